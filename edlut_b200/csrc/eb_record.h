// Device sort of the spike recording buffer (eb_record.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace eb {
// Words of the histogram workspace sort_record needs for n keys.
size_t record_sort_hist_words(int64_t n);
// Sort n records (step << 32 | neuron), every step in (s_lo, s_hi] and every
// neuron below n_cells, ascending; `tmp` holds n keys, `hist` the words above.
// *sorted is `keys` or `tmp`, whichever holds the result.
cudaError_t sort_record(unsigned long long *keys, unsigned long long *tmp, uint32_t *hist, int64_t n,
                        int64_t s_lo, int64_t s_hi, int64_t n_cells, cudaStream_t st,
                        unsigned long long **sorted);
// Kernels sort_record launches for those arguments.
int record_sort_launches(int64_t n, int64_t s_lo, int64_t s_hi, int64_t n_cells);
}  // namespace eb
