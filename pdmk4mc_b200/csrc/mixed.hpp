// Host interface of the mixed-precision (tcgen05, int8-sliced) outgoing
// plane-wave pass, mixed.cu.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

namespace pdmk {

// One CTA of the mixed contraction: the 128-row M tile `pair` (rows
// [128 pair, 128 pair + 128)) of one box, or of one split-K chunk of a box,
// over the slots [s_begin, s_end). `tab` holds the chunk table blocks of
// those slots (ceil((s_end - s_begin) / chunk) blocks of mixed_table_bytes),
// shared by the range's tiles.
struct MixItem {
  double cx, cy, cz;  // box centre
  double dk;          // mode spacing of the box's level
  int X, Y, Z;        // integer box coordinates at its level
  int M;              // decentring multiplier: 1 for levels >= 2, 3 for the root
  int s_begin, s_end;
  int pair;
  int pad_;
  double2* out;             // the box's H complex outputs (or its split-K partial)
  const unsigned char* tab;  // the range's chunk table blocks
};

// CTAs per box for n modes per axis half
int mixed_pairs(int nk);
// particles per pipeline chunk of the mixed pass for n modes per axis half
int mixed_chunk(int nk);
// bytes of one chunk's table block (a multiple of 16)
int mixed_table_bytes(int nk);
// 2-D tensor map over the slot arrays x, y, z, q (stride slot_capacity, which
// must be even), in boxes of kcp + 2 slots
void make_coord_map(CUtensorMap* map, const double* sx, int slot_capacity, int kcp);
// max |q| over n charges into *out (one block)
void launch_absmax(const double* sq, int n, double* out, cudaStream_t st);
// the mixed pass over device-resident lists: the table pass over nchunks
// (item, chunk) pairs (the item of a range's first tile, its chunk index),
// then the contraction over nitems tile items
void dispatch_mixed(int nk, const CUtensorMap& tmap, const MixItem* d_items, int nitems, const int2* d_chunks,
                    int nchunks, const double* d_qmax, int* d_err, cudaStream_t st);

}  // namespace pdmk
