// Level schedule of the samplers (sampling.h LevelSchedule). Written by
// potreeconverter_b200/autotune.py from a sweep on the target GPU; the
// values below are the sweep's best for the benchmarked workload, or the
// hand-set defaults until a sweep has run.
#pragma once
#define PCG_TUNED_CTA_MIN 8192
#define PCG_TUNED_SMALL_LEVEL_CTA_MIN 1024
#define PCG_TUNED_CLUSTER_MIN 131072
#define PCG_TUNED_WARP_BLOCKS_PER_SM 32
