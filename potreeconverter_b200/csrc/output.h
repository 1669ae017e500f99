// Output-stage and partition launchers.
#pragma once

#include "dev.h"

namespace pcg {

struct PayloadItem {        // one completed node with points
	const uint32_t* ids;
	const uint64_t* cols;    // packed colours or null
	int64_t count;
	int64_t out_offset;      // in points
};

// items: host copy of d_items (payloads in completion order, contiguous)
void launch_write_payloads(const DecodeParams& p, const std::vector<PayloadItem>& items, const PayloadItem* d_items, uint8_t* out,
                           DeviceMem& mem);
// Packed colour (r | g << 16 | b << 32) of every point's output record.
void launch_fill_colors(const DecodeParams& p, const uint32_t* ids, int64_t n, uint64_t* cols, DeviceMem& mem);
void launch_gather_u32(const uint32_t* src, const int64_t* idx, int64_t n, uint32_t* dst, DeviceMem& mem);
// Stable split of candidates by accepted flag: pre = exclusive prefix of the
// flags (n + 1 entries), accepted ids (and colours, records) compacted in
// order into acc_ids (acc_cols, acc_rec), rejected ids into rej_ids (skipped
// when null).
void launch_split(const uint8_t* accepted, int64_t n, const uint32_t* ids, const uint64_t* cols, const int4* rec, uint32_t* pre,
                  uint32_t* acc_ids, uint64_t* acc_cols, int4* acc_rec, uint32_t* rej_ids, DeviceMem& mem);

}  // namespace pcg
