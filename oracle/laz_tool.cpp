// ORACLE -- test infrastructure only. Writes LAZ files with the reference's
// vendored LASzip (Converter/libs/laszip, LASzip 3.4r3), the library the
// reference reads .laz inputs with (chunker_countsort_laszip.cpp:194-203,
// 750-772), so that the LAZ decode tests have inputs made by the reference's
// own code:
//
//   laz_tool compress <in.las> <out.laz> [chunk_size]
//   laz_tool decompress <in.laz> <out.las>
//
// Built by oracle/Makefile (target laz_tool) into oracle/_ref/.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "laszip/laszip_api.h"

static int fail(laszip_POINTER p, const char* what) {
	laszip_CHAR* msg = nullptr;
	if (p) laszip_get_error(p, &msg);
	fprintf(stderr, "%s: %s\n", what, msg ? msg : "(no message)");
	return 1;
}

static int copy(const char* in, const char* out, bool compress, unsigned chunk_size) {
	laszip_POINTER reader = nullptr, writer = nullptr;
	if (laszip_create(&reader)) return fail(nullptr, "create reader");
	laszip_BOOL is_compressed = 0;
	if (laszip_open_reader(reader, in, &is_compressed)) return fail(reader, "open reader");
	laszip_header* header = nullptr;
	if (laszip_get_header_pointer(reader, &header)) return fail(reader, "header");
	laszip_point* point = nullptr;
	if (laszip_get_point_pointer(reader, &point)) return fail(reader, "point");
	if (laszip_create(&writer)) return fail(nullptr, "create writer");
	if (laszip_set_header(writer, header)) return fail(writer, "set header");
	if (compress && chunk_size && laszip_set_chunk_size(writer, chunk_size)) return fail(writer, "chunk size");
	if (laszip_open_writer(writer, out, compress ? 1 : 0)) return fail(writer, "open writer");
	const long long n = header->extended_number_of_point_records > header->number_of_point_records
	                        ? (long long)header->extended_number_of_point_records
	                        : (long long)header->number_of_point_records;
	for (long long i = 0; i < n; i++) {
		if (laszip_read_point(reader)) return fail(reader, "read point");
		if (laszip_set_point(writer, point)) return fail(writer, "set point");
		if (laszip_write_point(writer)) return fail(writer, "write point");
	}
	if (laszip_close_writer(writer)) return fail(writer, "close writer");
	laszip_destroy(writer);
	laszip_close_reader(reader);
	laszip_destroy(reader);
	return 0;
}

int main(int argc, char** argv) {
	if (argc >= 4 && std::string(argv[1]) == "compress")
		return copy(argv[2], argv[3], true, argc >= 5 ? (unsigned)strtoul(argv[4], nullptr, 10) : 0u);
	if (argc >= 4 && std::string(argv[1]) == "decompress") return copy(argv[2], argv[3], false, 0u);
	fprintf(stderr, "usage: laz_tool compress <in.las> <out.laz> [chunk_size] | decompress <in.laz> <out.las>\n");
	return 2;
}
