// Internal interfaces of sort.cu.
#pragma once

#include "pmb_common.cuh"

namespace pmb {
int64_t radix_scratch_bytes(int64_t n);
int sort_by_cell(const int16_t* pmid, const float* disp, int64_t n, Mesh3 m, float cell, uint32_t* keys_out,
                 uint32_t* perm_out, void* scratch, cudaStream_t s);
}  // namespace pmb
