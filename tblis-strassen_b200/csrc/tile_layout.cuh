// Shared-memory (and packed-operand) tile layout of the DMMA kernels.
#pragma once

namespace tsb {

// Shared-memory layout of a k-major tile row (k fixed, m = 0..BM-1):
// inside each group of 16 rows the 8-byte slots form 8 pairs; rows g and g+8
// share pair (g + c(k)) mod 8, with c(k) = 2*(k mod 4) + (k/4 mod 2).  Then
//   * a fragment read (lanes g = 0..7, t = 0..3 reading rows g, g+8 of k-row
//     k4+t as one 128-bit pair) touches 8 distinct pairs per quarter warp;
//   * a cp.async write of 16 lanes covering 8 consecutive k of rows m, m+8
//     (k-fast loader) or 16 consecutive rows of one k (row-fast loader)
//     touches 16 distinct 8-byte slots of one 128-byte line.
__host__ __device__ __forceinline__ int swz_c(int k)
{
    return 2 * (k & 3) + ((k >> 2) & 1);
}

__host__ __device__ __forceinline__ int tile_pos(int k, int m, int ld)
{
    return k * ld + (m & ~15) + 2 * (((m & 7) + swz_c(k)) & 7) + ((m >> 3) & 1);
}

// Loader lane maps: element e (= thread + x * threads) of a BK x BM tile.
// k-fast: half-warps take 8 consecutive k of rows (m, m+8); row-fast: 16
// consecutive rows of one k.  Both write 16 distinct 8-byte slots of one
// 128-byte line per half-warp in the tile_pos layout.
template <int BK, int BM>
__device__ __forceinline__ void lane_map(bool kfast, int e, int& kk, int& m)
{
    if (kfast)
    {
        kk = (e & 7) + 8 * ((e >> 4) % (BK / 8));
        const int ridx = 2 * (e / (16 * (BK / 8))) + ((e >> 3) & 1);
        m = (ridx & ~15) | ((ridx & 1) << 3) | ((ridx >> 1) & 7);
    }
    else
    {
        m = e % BM;
        kk = e / BM;
    }
}

}  // namespace tsb
