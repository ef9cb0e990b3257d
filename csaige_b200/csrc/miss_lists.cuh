// Missing-call lists of a GRM handle, for the one-column products on the CUDA cores.
#pragma once
#include "engine.cuh"

namespace saige {

// The missing calls (code 01) of a handle's packed rows, grouped the way the one-column
// kernels walk the codes, so that a thread block reads the calls of the chunk it holds
// in shared memory as one contiguous segment.
//   pass A (block = a_rows marker rows, chunk = a_chunk_words words of 16 samples):
//     segment (block b, chunk c) = a_ent[a_seg[b a_nch + c] .. a_seg[b a_nch + c + 1]),
//     each entry (row in block) << a_bits | (sample in chunk);
//   pass B (block = b_rows samples, chunk = b_chunk marker rows):
//     segment (block p, chunk c) = b_ent[b_seg[p b_nch + c] .. ), each entry
//     (sample in block) << b_bits | (marker row in chunk).
// A one-column product sums its quantised vector over them exactly in int64 in place of
// the dense missing-flag sums: the same integers, so the same products to the bit.
struct MissLists {
  DevBuf a_ent, a_seg, b_ent, b_seg;
  int64_t a_nch = 0, b_nch = 0;
  int a_bits = 0, b_bits = 0;
  int state = 0;      // 0 not built, 1 built, -1 declined (the flag sums stay)
  int64_t total = 0;  // missing calls listed
};

// The lists are declined above this fraction of missing calls among the m x n entries:
// they would take more memory than a copy of the codes (8 bytes per missing call
// against 1/4 byte per entry), and the dense flag sums cost no more per entry there.
constexpr double kMissListMaxFrac = 0.03;

// How the one-column kernels take the codes (powers of two; a_rows divides m_pad, b_rows
// is two sample tiles and b_chunk a multiple of the 128-marker tiles).
struct MissShape {
  int a_rows;             // pass A: marker rows per block
  int64_t a_chunk_words;  // pass A: words of 16 samples per chunk
  int b_rows;             // pass B: samples per block (two 128-sample tiles)
  int64_t b_chunk;        // pass B: marker rows per chunk
};

// Builds L from h->geno and the sample-major tiles (tiles_s, s_ld marker tiles per
// sample tile) on st, synchronising st.  Too many missing calls, or memory that cannot
// be had, decline the lists (L->state = -1) without an error.
Status miss_lists_build(saige_grm* h, const uint8_t* tiles_s, int64_t s_ld, const MissShape& sh,
                        MissLists* L, cudaStream_t st);

}  // namespace saige
