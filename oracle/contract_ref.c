/*
 * Test infrastructure only -- the oracle.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg use it, and only as the checker; the product
 * never calls it.
 *
 * Plain-C restatement of the reference's contraction semantics on strided
 * tensors, C = alpha * A * B + beta * C with index-label strings:
 *
 *   - label classes and the diagonal of repeated labels follow
 *     src/iface/3t/mult.cxx:21-126 and src/util/tensor.hpp:305-342: a label
 *     repeated inside one tensor addresses its diagonal (strides add);
 *   - labels only in A or only in B are summed, labels only in C broadcast,
 *     labels in all three are batch indices (mult_ref,
 *     src/internal/3t/mult.cxx:313-473);
 *   - the per-element loop is contract_ref, src/internal/3t/mult.cxx:100-165:
 *     temp = sum A*B; temp *= alpha; C = beta == 0 ? temp : temp + beta*C
 *     (C is not read when beta == 0).
 *
 * The sum is accumulated in long double (x87 80-bit) so the oracle is at
 * least as accurate as the reference's FP64 micro-kernel; its agreement with
 * the compiled reference is pinned by tests/test_oracle.py and the fixtures
 * under tests/golden/.
 *
 * Build: gcc -O2 -shared -fPIC -o oracle/liboracle.so oracle/contract_ref.c
 */
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#define ORACLE_MAX_LABELS 64

typedef struct
{
    char label;
    int64_t len;
    int in_c;
} label_info;

static int find_label(const label_info* L, int n, char c)
{
    for (int i = 0; i < n; i++) if (L[i].label == c) return i;
    return -1;
}

/* Returns 0 on success, 1 on a label with inconsistent extents, 2 on too many
 * labels. */
int oracle_contract_d(double alpha,
                      const double* A, unsigned ndim_A, const int64_t* len_A,
                      const int64_t* stride_A, const char* idx_A,
                      const double* B, unsigned ndim_B, const int64_t* len_B,
                      const int64_t* stride_B, const char* idx_B,
                      double beta,
                      double* C, unsigned ndim_C, const int64_t* len_C,
                      const int64_t* stride_C, const char* idx_C)
{
    label_info L[ORACLE_MAX_LABELS];
    int nl = 0;
    const unsigned nd[3] = {ndim_A, ndim_B, ndim_C};
    const int64_t* lens[3] = {len_A, len_B, len_C};
    const char* idx[3] = {idx_A, idx_B, idx_C};
    for (int t = 0; t < 3; t++)
        for (unsigned d = 0; d < nd[t]; d++)
        {
            int i = find_label(L, nl, idx[t][d]);
            if (i < 0)
            {
                if (nl == ORACLE_MAX_LABELS) return 2;
                L[nl].label = idx[t][d];
                L[nl].len = lens[t][d];
                L[nl].in_c = 0;
                i = nl++;
            }
            else if (L[i].len != lens[t][d])
            {
                return 1;
            }
            if (t == 2) L[i].in_c = 1;
        }

    /* Per label, the stride it contributes to each tensor (sum over repeats). */
    int64_t sA[ORACLE_MAX_LABELS], sB[ORACLE_MAX_LABELS], sC[ORACLE_MAX_LABELS];
    memset(sA, 0, sizeof sA); memset(sB, 0, sizeof sB); memset(sC, 0, sizeof sC);
    for (unsigned d = 0; d < ndim_A; d++) sA[find_label(L, nl, idx_A[d])] += stride_A[d];
    for (unsigned d = 0; d < ndim_B; d++) sB[find_label(L, nl, idx_B[d])] += stride_B[d];
    for (unsigned d = 0; d < ndim_C; d++) sC[find_label(L, nl, idx_C[d])] += stride_C[d];

    int out[ORACLE_MAX_LABELS], sum[ORACLE_MAX_LABELS];
    int no = 0, ns = 0;
    for (int i = 0; i < nl; i++)
    {
        if (L[i].len == 0 && L[i].in_c) return 0;   /* C is empty */
        if (L[i].in_c) out[no++] = i; else sum[ns++] = i;
    }
    int empty_sum = 0;
    for (int i = 0; i < ns; i++) if (L[sum[i]].len == 0) empty_sum = 1;

    int64_t oc[ORACLE_MAX_LABELS], sc[ORACLE_MAX_LABELS];
    memset(oc, 0, sizeof oc);
    for (;;)
    {
        int64_t offA = 0, offB = 0, offC = 0;
        for (int i = 0; i < no; i++)
        {
            offA += oc[i] * sA[out[i]];
            offB += oc[i] * sB[out[i]];
            offC += oc[i] * sC[out[i]];
        }
        long double temp = 0.0L;
        if (!empty_sum)
        {
            memset(sc, 0, sizeof sc);
            for (;;)
            {
                int64_t a = offA, b = offB;
                for (int i = 0; i < ns; i++)
                {
                    a += sc[i] * sA[sum[i]];
                    b += sc[i] * sB[sum[i]];
                }
                temp += (long double)A[a] * (long double)B[b];
                int d = 0;
                for (; d < ns; d++)
                {
                    if (++sc[d] < L[sum[d]].len) break;
                    sc[d] = 0;
                }
                if (d == ns) break;
            }
        }
        temp *= (long double)alpha;
        if (beta == 0.0) C[offC] = (double)temp;
        else C[offC] = (double)(temp + (long double)beta * (long double)C[offC]);

        int d = 0;
        for (; d < no; d++)
        {
            if (++oc[d] < L[out[d]].len) break;
            oc[d] = 0;
        }
        if (d == no) break;
    }
    return 0;
}
