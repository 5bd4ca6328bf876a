// Internal helpers of the .f0 reader shared by the cube job (host code).
#pragma once
#include <string>
#include <vector>
#include <cstdint>
#include "../../include/snapi_cuda.h"

namespace snapi_f0 {
// Header of an open file (ck_synch_hd + the first part of ana_fzread).
int parse(int fd, snapi_f0_info *info);
// Elements [first, first + count) converted to out_type (the file's type, FLOAT32 or FLOAT64).
int read_range(int fd, const snapi_f0_info &info, long long first, long long count, void *out, int out_type,
               std::vector<uint8_t> &scratch);
int type_size(int type);
void set_error(const std::string &msg);
}  // namespace snapi_f0
