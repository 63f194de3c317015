// HBM-bound helper kernels of the contraction path.
//
//   scale_kernel        C = beta*C (beta == 0: C = 0 without reading C) for
//                       alpha == 0 or an empty contracted range; replaces the
//                       set/scale branch of src/stra_iface/3t/stra_mult.cxx:215-231.
//   sum_gather_kernel   dense S = sum_t sign_t * X[block_t]: the explicit Strassen
//                       operand sums of the Naive variant (straprim_naive2,
//                       src/stra_internal/3t/straprim_common.hpp:70-157, which
//                       forms them with add() into S and T buffers).
//   scatter_add_kernel  C_q = (first ? beta*C_q : C_q) + sign_q*alpha*M for the
//                       C blocks of one product: the M -> C update of the AB and
//                       Naive variants (src/stra_internal/3t/straprim_common.hpp:
//                       156, 187-203, tensor2matrix.hpp:390-830).
//   combine_kernel      C_h = alpha * sum_p W[h][p] M_p + beta * C_h for every C
//                       block h at once, after the products have run side by
//                       side into their own M_p (the product-parallel schedule):
//                       each M_p is read once, C written once.
//
// The first three are grid-stride loops over (batch, row, col) with the column
// index fastest; the scatter vectors make the access pattern coalesced
// whenever the fastest C (or X) mode is the column bundle's first mode.
#include "kernels.cuh"
#include "timing.hpp"

#include <algorithm>
#include <atomic>

namespace tsb {

extern std::atomic<unsigned long long> g_launches;

namespace {

constexpr int THREADS = 256;

unsigned grid_for(int64_t total)
{
    int64_t blocks = (total + THREADS - 1) / THREADS;
    const int64_t cap = 148 * 16;   // 16 resident blocks per SM on 148 SMs
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return (unsigned)blocks;
}

__global__ void scale_f32_kernel(const ScaleF32Args a)
{
    const int64_t total = a.batch * a.m * a.n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t j = e % a.n;
        const int64_t rest = e / a.n;
        const int64_t i = rest % a.m;
        const int64_t b = rest / a.m;
        float* p = a.C + a.bC[b] + a.rsC[i] + a.csC[j];
        *p = (a.beta == 0.f) ? 0.f : a.beta * *p;
    }
}

__global__ void scale_kernel(const ScaleArgs a)
{
    const int64_t total = a.batch * a.m * a.n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t j = e % a.n;
        const int64_t rest = e / a.n;
        const int64_t i = rest % a.m;
        const int64_t b = rest / a.m;
        double* p = a.C + a.bC[b] + a.rsC[i] + a.csC[j];
        *p = (a.beta == 0.0) ? 0.0 : a.beta * *p;
    }
}

__global__ void sum_gather_kernel(const SumGatherArgs a)
{
    const int64_t total = a.batch * a.rows * a.cols;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t j = e % a.cols;
        const int64_t rest = e / a.cols;
        const int64_t i = rest % a.rows;
        const int64_t b = rest / a.rows;
        double v = 0.0;
        for (int t = 0; t < a.nt; t++)
        {
            const int64_t gi = a.t_r[t] * a.rows + i;
            const int64_t gj = a.t_c[t] * a.cols + j;
            if (gi < a.rows_full && gj < a.cols_full)
            {
                const double x = a.X[a.bX[b] + a.rsX[gi] + a.csX[gj]];
                v += a.t_s[t] < 0 ? -x : x;
            }
        }
        a.out[e] = v;
    }
}

__global__ void scatter_add_kernel(const ScatterAddArgs a)
{
    const int64_t total = a.batch * a.ms * a.ns;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t j = e % a.ns;
        const int64_t rest = e / a.ns;
        const int64_t i = rest % a.ms;
        const int64_t b = rest / a.ms;
        const double mv = a.M[e];
        for (int q = 0; q < a.nc; q++)
        {
            const int64_t gi = a.c_r[q] * a.ms + i;
            const int64_t gj = a.c_c[q] * a.ns + j;
            if (gi >= a.m || gj >= a.n) continue;
            double* p = a.C + a.bC[b] + a.rsC[gi] + a.csC[gj];
            const double coef = a.c_s[q] < 0 ? -a.alpha : a.alpha;
            double v = coef * mv;
            if (!a.c_first[q]) v += *p;
            else if (a.beta != 0.0) v += a.beta * *p;
            *p = v;
        }
    }
}

// One thread per local position (i, j) of every C block: it reads each
// product's M_p there once, adds it (with sign) into the accumulators of the
// product's block positions, kept in shared memory (column threadIdx.x of
// acc[h], H * H rows of dynamic shared memory), then writes the H * H C
// elements.  M is read once in total.
// Grid: x over the ms * ns local positions (fastest index that of M's
// layout), y over batch entries.
constexpr int COMBINE_THREADS = 256;

template <class T>
__global__ void __launch_bounds__(COMBINE_THREADS)
combine_kernel(const __grid_constant__ CombineArgsT<T> a)
{
    extern __shared__ double combine_acc[];
    double (*acc)[COMBINE_THREADS] = reinterpret_cast<double (*)[COMBINE_THREADS]>(combine_acc);
    const int tid = threadIdx.x;
    const int H = a.H, H2 = H * H;
    const uint32_t per = (uint32_t)(a.ms * a.ns);
    const uint32_t fast = (uint32_t)(a.col_major ? a.ms : a.ns);
    for (int64_t b = blockIdx.y; b < a.batch; b += gridDim.y)
    {
        const T* __restrict__ Mb = a.M + b * (int64_t)per;
        const int64_t cb = a.bC[b];
        for (uint32_t loc = blockIdx.x * COMBINE_THREADS + tid; loc < per; loc += gridDim.x * COMBINE_THREADS)
        {
            for (int h = 0; h < H2; h++) acc[h][tid] = 0.0;
            // seven products' loads in flight before their accumulator updates
            for (int p0 = 0; p0 < a.np; p0 += 7)
            {
                double x[7];
#pragma unroll
                for (int u = 0; u < 7; u++)
                    x[u] = p0 + u < a.np ? (double)__ldg(Mb + (p0 + u) * a.m_pstride + loc) : 0.0;
#pragma unroll
                for (int u = 0; u < 7; u++)
                {
                    const int p = p0 + u;
                    if (p >= a.np) break;
                    for (int t = 0; t < a.nt[p]; t++)
                        acc[a.th[p][t]][tid] += a.ts[p][t] < 0 ? -x[u] : x[u];
                }
            }
            const uint32_t q = loc / fast, r = loc - q * fast;
            const int64_t i = a.col_major ? r : q, j = a.col_major ? q : r;
            for (int hr = 0; hr < H; hr++)
            {
                const int64_t gi = hr * a.ms + i;
                if (gi >= a.m) break;
                const int64_t ro = cb + a.rsC[gi];
                for (int hc = 0; hc < H; hc++)
                {
                    const int64_t gj = hc * a.ns + j;
                    if (gj >= a.n) break;
                    T* p = a.C + ro + a.csC[gj];
                    const double v = acc[hr * H + hc][tid];
                    *p = (T)(a.beta != 0.0 ? a.alpha * v + a.beta * (double)*p : a.alpha * v);
                }
            }
        }
    }
}

}  // namespace

template <class T>
cudaError_t launch_combine_t(const CombineArgsT<T>& a, cudaStream_t stream)
{
    const int64_t per = a.ms * a.ns;
    if (per <= 0 || a.batch <= 0) return cudaSuccess;
    if (a.H < 1 || a.H > 4 || a.np < 1 || a.np > MAX_COMBINE_PRODUCTS ||
        per >= ((int64_t)1 << 32) - COMBINE_THREADS * (int64_t)65535)
        return cudaErrorInvalidValue;
    for (int p = 0; p < a.np; p++)
    {
        if (a.nt[p] < 0 || a.nt[p] > 4) return cudaErrorInvalidValue;
        for (int t = 0; t < a.nt[p]; t++)
            if (a.th[p][t] < 0 || a.th[p][t] >= a.H * a.H) return cudaErrorInvalidValue;
    }
    const dim3 grid((unsigned)std::min<int64_t>((per + COMBINE_THREADS - 1) / COMBINE_THREADS, 65535),
                    (unsigned)std::min<int64_t>(a.batch, 65535));
    const size_t smem = (size_t)a.H * a.H * COMBINE_THREADS * sizeof(double);
    // as much shared memory as the SM gives: occupancy is bound by it
    cudaError_t err = cudaFuncSetAttribute(combine_kernel<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                           (int)cudaSharedmemCarveoutMaxShared);
    if (err != cudaSuccess) return err;
    timing_begin(KK_AUX, stream);
    combine_kernel<T><<<grid, COMBINE_THREADS, smem, stream>>>(a);
    timing_end(KK_AUX, stream);
    err = cudaGetLastError();
    if (err == cudaSuccess) g_launches++;
    return err;
}

cudaError_t launch_combine(const CombineArgs& a, cudaStream_t stream) { return launch_combine_t(a, stream); }
cudaError_t launch_combine(const CombineF32Args& a, cudaStream_t stream) { return launch_combine_t(a, stream); }

cudaError_t launch_scale(const ScaleArgs& a, cudaStream_t stream)
{
    const int64_t total = a.batch * a.m * a.n;
    if (total <= 0) return cudaSuccess;
    timing_begin(KK_AUX, stream);
    scale_kernel<<<grid_for(total), THREADS, 0, stream>>>(a);
    timing_end(KK_AUX, stream);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) g_launches++;
    return err;
}

cudaError_t launch_scale_f32(const ScaleF32Args& a, cudaStream_t stream)
{
    const int64_t total = a.batch * a.m * a.n;
    if (total <= 0) return cudaSuccess;
    timing_begin(KK_AUX, stream);
    scale_f32_kernel<<<grid_for(total), THREADS, 0, stream>>>(a);
    timing_end(KK_AUX, stream);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) g_launches++;
    return err;
}

cudaError_t launch_sum_gather(const SumGatherArgs& a, cudaStream_t stream)
{
    const int64_t total = a.batch * a.rows * a.cols;
    if (total <= 0) return cudaSuccess;
    timing_begin(KK_AUX, stream);
    sum_gather_kernel<<<grid_for(total), THREADS, 0, stream>>>(a);
    timing_end(KK_AUX, stream);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) g_launches++;
    return err;
}

cudaError_t launch_scatter_add(const ScatterAddArgs& a, cudaStream_t stream)
{
    const int64_t total = a.batch * a.ms * a.ns;
    if (total <= 0) return cudaSuccess;
    if (a.nc < 0 || a.nc > 4) return cudaErrorInvalidValue;
    timing_begin(KK_AUX, stream);
    scatter_add_kernel<<<grid_for(total), THREADS, 0, stream>>>(a);
    timing_end(KK_AUX, stream);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) g_launches++;
    return err;
}

}  // namespace tsb
