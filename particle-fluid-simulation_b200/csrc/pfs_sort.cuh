// pfs_sort.cuh — stable LSD radix sort of (cell key, slot) pairs.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace pfs {

// Bits a key < n can occupy, and the 8-bit passes that covers.
int sort_key_bits(uint32_t n);
int sort_passes(uint32_t n);
uint32_t sort_tiles(uint32_t n);
// Words of scratch the per-tile histograms need for n keys.
size_t sort_hist_words(uint32_t n);
// Kernel launches one sort issues.
int sort_launches(uint32_t n);

// Stable sort of keys_in[0..n) (values = slot index) into keys_out/vals_out.
// key_bits: bits that can be non-zero (sort_key_bits(n) for one table).
// Scratch: keys_tmp/vals_tmp (n words each), hist (sort_hist_words(n)),
// digit_total (256 words).  err: device error word.
cudaError_t sort_pairs(const uint32_t* keys_in, uint32_t n, int key_bits, uint32_t* keys_out,
                       uint32_t* vals_out, uint32_t* keys_tmp, uint32_t* vals_tmp,
                       uint32_t* hist, uint32_t* digit_total, uint32_t* err,
                       cudaStream_t stream);

}  // namespace pfs
