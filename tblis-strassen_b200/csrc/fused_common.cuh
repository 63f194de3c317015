// Geometry and device helpers shared by the two forms of the fused FP64
// Strassen kernel (fused_kernel.cu: gathers through the scatter vectors;
// fused_tma.cu: tensor-map copies of tiles that are boxes of the operands).
#pragma once

#include "kernels.cuh"

#include <cstdint>

namespace tsb {
namespace fused {

constexpr int FT = 128;                  // tile rows (A side) and columns (B side)
constexpr int FSTAGES = 3;
constexpr int FHMAX = 4;                 // largest block grid side (level 2)
constexpr int NPW = 4;                   // producer warps (one warpgroup)
constexpr int NCW = 8;                   // consumer warps: 2 (M) x 4 (N)
constexpr int FTHREADS = 32 * (NPW + NCW);
constexpr int PT = 32 * NPW;             // producer threads
constexpr int CT = 32 * NCW;             // consumer threads
constexpr int CWM = 2, CWN = 4;
constexpr int WTM = FT / CWM, WTN = FT / CWN;   // 64 x 32 warp tile
constexpr int MI = WTM / 16, NI = WTN / 8;      // 4 x 4 fragments

struct FusedCtrl
{
    uint64_t full[FSTAGES], empty[FSTAGES];
    int abort;
};

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0)
{
    asm("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 "
        "{%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

// Named barrier `id` over `count` threads with an OR over `flag`.
template <int ID, int COUNT>
__device__ __forceinline__ bool bar_any(bool flag)
{
    uint32_t out;
    asm volatile("{\n.reg .pred q, p;\nsetp.ne.u32 q, %1, 0;\nbar.red.or.pred p, %2, %3, q;\n"
                 "selp.u32 %0, 1, 0, p;\n}\n" : "=r"(out) : "r"((uint32_t)flag), "n"(ID), "n"(COUNT) : "memory");
    return out != 0;
}

template <int ID, int COUNT>
__device__ __forceinline__ void bar_sync()
{
    asm volatile("bar.sync %0, %1;\n" :: "n"(ID), "n"(COUNT) : "memory");
}

// Work item w -> (batch b, row tile tm, column tile tn): groups of 8 row tiles
// walk the column tiles together so concurrent CTAs share panels in L2.
__device__ __forceinline__ void decode_work(const DmmaArgs& a, int64_t w, int64_t& b, int64_t& tm, int64_t& tn)
{
    const int64_t tiles = (int64_t)a.tiles_m * a.tiles_n;
    b = w / tiles;
    const int64_t tw = w - b * tiles;
    const int64_t GROUP = 8;
    const int64_t group = tw / (GROUP * a.tiles_n);
    const int64_t first_m = group * GROUP;
    const int64_t gsize = (a.tiles_m - first_m) < GROUP ? (a.tiles_m - first_m) : GROUP;
    tm = first_m + (tw % gsize);
    tn = (tw % (GROUP * a.tiles_n)) / gsize;
}

// The C tables of a work item: offsets of the tile's rows (columns) in every
// block row (column) h of the C grid, OFF_INVALID past the extents.  Written
// by the consumer threads (ctid < CT).
__device__ __forceinline__ void fill_c_tables(const DmmaArgs& a, int64_t b, int64_t tm, int64_t tn,
                                              int64_t* rowC, int64_t* colC, int ctid)
{
    const int H = a.H;
    const int Hn = a.Hn > 0 ? a.Hn : a.H;
    const int64_t offC = a.bC[b];
    for (int i = ctid; i < FHMAX * FT; i += CT)
    {
        const int h = i / FT, r = i % FT;
        const int64_t li = tm * FT + r, gi = h * a.ms + li;
        rowC[i] = (h < H && li < a.ms && gi < a.m) ? offC + a.rsC[gi] : OFF_INVALID;
        const int64_t lj = tn * FT + r, gj = h * a.ns + lj;
        colC[i] = (h < Hn && lj < a.ns && gj < a.n) ? a.csC[gj] : OFF_INVALID;
    }
}

// Epilogue of one product: C_t = (first ? beta*C_t : C_t) + coef_t*acc for
// the product's C blocks t, with coef_t = +-alpha (sign_t, times -1 when
// `lead_neg`: the signs of the first blocks of the operand sums, when the
// consumer formed the sums as A_0 +- A_1).  Fragment row g (+8) of warp row
// block mi is tile row wm + 16 mi + row8[g] (+8); fragment column c of
// column block ni is tile column wn + 8 ni + col8[c].  Loads of a row are
// issued before its stores.
__device__ __forceinline__ void product_epilogue(const DmmaArgs& a, const DevProduct& P, bool lead_neg,
                                                 const int64_t* rowC, const int64_t* colC,
                                                 const double (&acc)[MI][NI][4], int wm, int wn,
                                                 int row_g, int col0, int col1)
{
    for (int t = 0; t < P.nc; t++)
    {
        const int64_t* rt = rowC + P.c_r[t] * FT;
        const int64_t* ct = colC + P.c_c[t] * FT;
        const double coef = ((P.c_s[t] < 0) != lead_neg) ? -a.alpha : a.alpha;
        const bool first = P.c_first[t] != 0;
        const bool read_c = !first || a.beta != 0.0;
        const double cb = first ? a.beta : 1.0;
#pragma unroll
        for (int mi = 0; mi < MI; mi++)
#pragma unroll
            for (int hr = 0; hr < 2; hr++)
            {
                const int64_t ro = rt[wm + mi * 16 + row_g + hr * 8];
                if (ro == OFF_INVALID) continue;
                double cv[NI][2];
#pragma unroll
                for (int ni = 0; ni < NI; ni++)
#pragma unroll
                    for (int hc = 0; hc < 2; hc++)
                    {
                        const int64_t co = ct[wn + ni * 8 + (hc ? col1 : col0)];
                        cv[ni][hc] = (read_c && co != OFF_INVALID) ? a.C[ro + co] : 0.0;
                    }
#pragma unroll
                for (int ni = 0; ni < NI; ni++)
#pragma unroll
                    for (int hc = 0; hc < 2; hc++)
                    {
                        const int64_t co = ct[wn + ni * 8 + (hc ? col1 : col0)];
                        if (co == OFF_INVALID) continue;
                        a.C[ro + co] = coef * acc[mi][ni][hr * 2 + hc] + cb * cv[ni][hc];
                    }
            }
    }
}

}  // namespace fused
}  // namespace tsb
