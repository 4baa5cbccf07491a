// host_io.h — host-side LIME/ILDG container codec and input-file parser (no CUDA).
#pragma once
#include <stdint.h>
#include <stdio.h>

#include <string>

#include "../../include/qcb.h"

namespace qcb {

// LIME record header: 144 bytes, big-endian (SciDAC LIME format): magic 0x456789ab (u32),
// version 1 (u16), flags (u16; bit 15 = message begin, bit 14 = message end), data length
// (u64), record type (128 bytes, NUL padded).  Record data is padded to a multiple of 8.
constexpr uint32_t LIME_MAGIC = 0x456789abu;
constexpr size_t LIME_HDR = 144;

bool lime_write_header(FILE* fp, bool mb, bool me, const char* type, uint64_t nbytes);
bool lime_write_padding(FILE* fp, uint64_t nbytes);
// Scan records for `type`; on success *offset = file offset of its data, *nbytes = length.
// Returns 0 on success, QCB_ERR_FORMAT for a malformed file, QCB_ERR_IO if absent.
int lime_find(FILE* fp, const char* type, uint64_t* offset, uint64_t* nbytes, std::string* err);

// ILDG "ildg-format" XML record body (reference: generate_ildg_xml, src/io/ildg.cpp:13-22).
std::string ildg_xml(const int dims[4]);

// Input-file parsers (semantics in host_io.cpp); p must hold the defaults on entry.
int params_load(const char* path, qcb_hb_params* p, std::string* err);
int ecmc_params_load(const char* path, qcb_ecmc_run_params* p, std::string* err);

}  // namespace qcb
