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
// Words of scratch a sort of n keys of key_bits bits needs (digit
// histograms, tile counters and look-back words).
size_t sort_scratch_words(uint32_t n, int key_bits);
// Kernel launches one sort issues (plus one memset).
int sort_launches(uint32_t n);

// Stable sort of keys_in[0..n) (values = slot index) into keys_out/vals_out.
// key_bits: bits that can be non-zero (sort_key_bits(n) for one table; at
// most 32).  Scratch: keys_tmp/vals_tmp (n words each), scratch
// (sort_scratch_words(n, key_bits)); none of them may overlap the inputs or
// outputs.  err: device error word.
cudaError_t sort_pairs(const uint32_t* keys_in, uint32_t n, int key_bits, uint32_t* keys_out,
                       uint32_t* vals_out, uint32_t* keys_tmp, uint32_t* vals_tmp,
                       uint32_t* scratch, uint32_t* err, cudaStream_t stream);

}  // namespace pfs
