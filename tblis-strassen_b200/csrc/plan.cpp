// Contraction planning (see plan.hpp for the reference behaviour followed).
#include "plan.hpp"

#include <algorithm>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

namespace tsb {

namespace {

// Mode list of one tensor after diagonal(): label, extent, stride.
struct Mode { label_type idx; int64_t len; int64_t stride; };

// diagonal(), src/util/tensor.hpp:305-342: sort modes by label, merge a
// repeated label into one mode whose stride is the sum (the extents must agree),
// drop extent-1 modes.
int diagonal(const tblis_tensor* T, const label_type* idx, std::vector<Mode>& out)
{
    out.clear();
    std::vector<unsigned> order(T->ndim);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](unsigned a, unsigned b) { return idx[a] < idx[b]; });
    for (unsigned pos = 0; pos < T->ndim; pos++)
    {
        unsigned d = order[pos];
        int64_t len = T->len[d];
        if (len < 0) return TBLIS_STRA_ERR_ARG;
        if (pos > 0 && idx[d] == idx[order[pos - 1]])
        {
            // repeated label: extents must agree; strides add
            unsigned p = order[pos - 1];
            if (T->len[p] != len) return TBLIS_STRA_ERR_EXTENT;
            if (len != 1)
            {
                if (out.empty() || out.back().idx != idx[d]) return TBLIS_STRA_ERR_EXTENT;
                out.back().stride += T->stride[d];
            }
            continue;
        }
        if (len != 1) out.push_back({idx[d], len, (int64_t)T->stride[d]});
    }
    return TBLIS_STRA_SUCCESS;
}

const Mode* find(const std::vector<Mode>& v, label_type l)
{
    for (auto& m : v) if (m.idx == l) return &m;
    return nullptr;
}

// fold(), src/util/tensor.hpp:270-303: order modes by the first tensor's stride,
// then merge mode i into the previous one when it is contiguous with it in
// every tensor of the class.
void fold(Bundle& b)
{
    const size_t nd = b.len.size();
    if (nd == 0) return;
    const size_t nt = b.stride.size();
    std::vector<size_t> order(nd);
    std::iota(order.begin(), order.end(), size_t(0));
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
        return b.stride[0][x] < b.stride[0][y];
    });
    Bundle out;
    out.stride.resize(nt);
    for (size_t i = 0; i < nd; i++)
    {
        size_t d = order[i];
        bool contiguous = false;
        if (i != 0)
        {
            size_t p = order[i - 1];
            contiguous = true;
            for (size_t t = 0; t < nt; t++)
                if (b.stride[t][d] != b.stride[t][p] * b.len[p]) contiguous = false;
        }
        if (contiguous)
        {
            out.len.back() *= b.len[d];
        }
        else
        {
            out.idx.push_back(b.idx[d]);
            out.len.push_back(b.len[d]);
            for (size_t t = 0; t < nt; t++) out.stride[t].push_back(b.stride[t][d]);
        }
    }
    b = std::move(out);
}

// Reorder a bundle's modes by ascending |stride| of the given tensors in
// priority order (the reference's sort_by_stride(stride_C_AC, stride_A_AC),
// src/stra_internal/3t/stra_mult.cxx:336-338), so that flat index 0,1,2...
// walks the fastest mode first.
void sort_modes(Bundle& b, std::vector<int> prio)
{
    const size_t nd = b.len.size();
    std::vector<size_t> order(nd);
    std::iota(order.begin(), order.end(), size_t(0));
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
        for (int t : prio)
        {
            int64_t sx = std::llabs(b.stride[t][x]), sy = std::llabs(b.stride[t][y]);
            if (sx != sy) return sx < sy;
        }
        return false;
    });
    Bundle out;
    out.stride.resize(b.stride.size());
    for (size_t d : order)
    {
        out.idx.push_back(b.idx[d]);
        out.len.push_back(b.len[d]);
        for (size_t t = 0; t < b.stride.size(); t++) out.stride[t].push_back(b.stride[t][d]);
    }
    b = std::move(out);
}

int64_t prod_len(const std::vector<int64_t>& len)
{
    int64_t p = 1;
    for (int64_t l : len) p *= l;
    return p;
}

// Flattened offsets of every index of a mode list (fastest mode first).
void scatter(const std::vector<int64_t>& len, const std::vector<int64_t>& stride,
             std::vector<int64_t>& out)
{
    int64_t total = prod_len(len);
    out.assign((size_t)total, 0);
    if (total == 0) return;
    std::vector<int64_t> digit(len.size(), 0);
    int64_t off = 0;
    for (int64_t i = 0; i < total; i++)
    {
        out[(size_t)i] = off;
        for (size_t d = 0; d < len.size(); d++)
        {
            digit[d]++;
            off += stride[d];
            if (digit[d] < len[d]) break;
            off -= stride[d] * len[d];
            digit[d] = 0;
        }
    }
}

// Append the modes of `src` (with strides for tensors listed in `map`, a
// missing tensor getting stride 0) to `dst` whose tensors are `dst_tensors`.
void append_modes(std::vector<int64_t>& len, std::vector<std::vector<int64_t>>& strides,
                  const Bundle& src, const std::vector<int>& src_slot_for_dst)
{
    for (size_t d = 0; d < src.len.size(); d++)
    {
        len.push_back(src.len[d]);
        for (size_t t = 0; t < strides.size(); t++)
        {
            int s = src_slot_for_dst[t];
            strides[t].push_back(s < 0 ? 0 : src.stride[(size_t)s][d]);
        }
    }
}

// Smallest |stride| among the first `lead` modes of extent > 1 (0 if none):
// the stride consecutive loader threads walk inside one k-step.
int64_t first_stride(const std::vector<int64_t>& len, const std::vector<int64_t>& stride,
                     int lead = 1)
{
    int64_t best = 0;
    int seen = 0;
    for (size_t d = 0; d < len.size() && seen < lead; d++)
    {
        if (len[d] <= 1) continue;
        int64_t s = std::llabs(stride[d]);
        if (seen == 0 || s < best) best = s;
        seen++;
    }
    return best;
}

// Contracted-index order for two operands whose fastest modes differ.
//
// The order of the contracted index set is free: any bijection gives the same
// sum, and Strassen's halving is valid for any split of the index set into
// equal parts.  When A's smallest-stride mode dA and B's smallest-stride mode
// dB differ (e.g. A(e,f,..) and B(f,..,e) column-major: A runs along e, B
// along f), a plain order leaves one operand with no contiguous run inside a
// k-step.  This splits dA into (a, len/a) and dB into (b, len/b) and puts the
// two short parts first, so every aligned chunk of a*b consecutive indices is
// an a x b box: A reads runs of a elements and B runs of b elements (a = b =
// one 32-byte sector: 4 x 4 = 16 for FP64, 8 x 8 = 64 for FP32, the k-steps
// of the kernels).  Returns whether the order was changed.
bool block_interleave(std::vector<int64_t>& len, std::vector<std::vector<int64_t>>& str, int run)
{
    const size_t nd = len.size();
    if (nd < 2) return false;
    auto smallest = [&](int t) {
        size_t best = nd;
        for (size_t d = 0; d < nd; d++)
            if (len[d] > 1 && (best == nd || std::llabs(str[t][d]) < std::llabs(str[t][best]))) best = d;
        return best;
    };
    const size_t dA = smallest(0), dB = smallest(1);
    if (dA == nd || dB == nd || dA == dB) return false;
    if (std::llabs(str[0][dA]) != 1 || std::llabs(str[1][dB]) != 1) return false;
    // Runs of `run` elements = one 32-byte sector (4 doubles, 8 floats).
    const int choices[][2] = {{run, run}, {run, run / 2}, {run / 2, run}, {run / 2, run / 2}, {2, 2}};
    for (auto& c : choices)
    {
        const int64_t a = c[0], b = c[1];
        if (a < 2 || b < 2) continue;
        if (len[dA] % a || len[dB] % b || len[dA] == a || len[dB] == b) continue;
        std::vector<int64_t> nl;
        std::vector<std::vector<int64_t>> ns(str.size());
        auto push = [&](int64_t l, size_t d, int64_t mult) {
            nl.push_back(l);
            for (size_t t = 0; t < str.size(); t++) ns[t].push_back(str[t][d] * mult);
        };
        push(a, dA, 1);
        push(b, dB, 1);
        push(len[dA] / a, dA, a);
        push(len[dB] / b, dB, b);
        for (size_t d = 0; d < nd; d++)
            if (d != dA && d != dB) push(len[d], d, 1);
        len = nl;
        str = ns;
        return true;
    }
    return false;
}

}  // namespace

void tensor_span(unsigned ndim, const len_type* len, const stride_type* stride,
                 int64_t& lo, int64_t& hi)
{
    lo = 0; hi = 0;
    for (unsigned d = 0; d < ndim; d++)
    {
        if (len[d] == 0) { lo = 0; hi = -1; return; }
        int64_t ext = (int64_t)(len[d] - 1) * (int64_t)stride[d];
        if (ext < 0) lo += ext; else hi += ext;
    }
}

int plan_contraction(const tblis_tensor* A, const label_type* idx_A,
                     const tblis_tensor* B, const label_type* idx_B,
                     const tblis_tensor* C, const label_type* idx_C,
                     GemmView& g, bool build_scatter)
{
    if (!A || !B || !C) return TBLIS_STRA_ERR_NULL;
    const tblis_tensor* T[3] = {A, B, C};
    const label_type* I[3] = {idx_A, idx_B, idx_C};
    for (int t = 0; t < 3; t++)
    {
        if (T[t]->ndim > 0 && (!I[t] || !T[t]->len || !T[t]->stride)) return TBLIS_STRA_ERR_NULL;
        if (T[t]->ndim > 64) return TBLIS_STRA_ERR_ARG;
    }
    if (A->type != B->type || A->type != C->type) return TBLIS_STRA_ERR_TYPE;
    if (A->type != TYPE_DOUBLE && A->type != TYPE_FLOAT) return TBLIS_STRA_ERR_TYPE;
    if (A->conj || B->conj || C->conj) return TBLIS_STRA_ERR_CONJ;

    g = GemmView();
    g.type = A->type;
    if (A->type == TYPE_DOUBLE)
    {
        double a, b, c;
        std::memcpy(&a, A->scalar, 8); std::memcpy(&b, B->scalar, 8); std::memcpy(&c, C->scalar, 8);
        g.alpha = a * b; g.beta = c;
    }
    else
    {
        float a, b, c;
        std::memcpy(&a, A->scalar, 4); std::memcpy(&b, B->scalar, 4); std::memcpy(&c, C->scalar, 4);
        g.alpha = (double)(a * b); g.beta = (double)c;
    }

    std::vector<Mode> M[3];
    for (int t = 0; t < 3; t++)
    {
        int st = diagonal(T[t], I[t], M[t]);
        if (st) return st;
        tensor_span(T[t]->ndim, T[t]->len, T[t]->stride, g.lo[t], g.hi[t]);
    }

    // Label classes (src/iface/3t/mult.cxx:43-86) with the extent checks of
    // its TBLIS_ASSERTs turned into a status.
    std::vector<label_type> labels;
    for (int t = 0; t < 3; t++) for (auto& m : M[t]) labels.push_back(m.idx);
    std::sort(labels.begin(), labels.end());
    labels.erase(std::unique(labels.begin(), labels.end()), labels.end());

    g.ABC.stride.resize(3); g.AB.stride.resize(2); g.AC.stride.resize(2);
    g.BC.stride.resize(2); g.A_only.stride.resize(1); g.B_only.stride.resize(1);
    g.C_only.stride.resize(1);
    for (label_type l : labels)
    {
        const Mode* ma = find(M[0], l);
        const Mode* mb = find(M[1], l);
        const Mode* mc = find(M[2], l);
        int64_t len = ma ? ma->len : mb ? mb->len : mc->len;
        if ((ma && ma->len != len) || (mb && mb->len != len) || (mc && mc->len != len))
            return TBLIS_STRA_ERR_EXTENT;
        Bundle* b; std::vector<const Mode*> ms;
        if (ma && mb && mc) { b = &g.ABC; ms = {ma, mb, mc}; }
        else if (ma && mb)  { b = &g.AB;  ms = {ma, mb}; }
        else if (ma && mc)  { b = &g.AC;  ms = {ma, mc}; }
        else if (mb && mc)  { b = &g.BC;  ms = {mb, mc}; }
        else if (ma)        { b = &g.A_only; ms = {ma}; }
        else if (mb)        { b = &g.B_only; ms = {mb}; }
        else                { b = &g.C_only; ms = {mc}; }
        b->idx.push_back(l);
        b->len.push_back(len);
        for (size_t t = 0; t < ms.size(); t++) b->stride[t].push_back(ms[t]->stride);
    }

    // fold() each class (src/iface/3t/mult.cxx:120-126).
    fold(g.ABC); fold(g.AB); fold(g.AC); fold(g.BC);
    fold(g.A_only); fold(g.B_only); fold(g.C_only);

    // Flattening order (src/stra_internal/3t/stra_mult.cxx:336-338):
    // AC by (C, A) stride, BC by (C, B), AB by (A, B); batch by (C, A, B).
    sort_modes(g.AC, {1, 0});
    sort_modes(g.BC, {1, 0});
    sort_modes(g.AB, {0, 1});
    sort_modes(g.ABC, {2, 0, 1});

    // Rows: AC.  Columns: BC.  Contracted: AB + A-only (B stride 0) + B-only
    // (A stride 0).  Batch: ABC + C-only (A, B stride 0).
    std::vector<int64_t> k_len = g.AB.len;
    std::vector<std::vector<int64_t>> k_str = {g.AB.stride[0], g.AB.stride[1]};
    append_modes(k_len, k_str, g.A_only, {0, -1});
    append_modes(k_len, k_str, g.B_only, {-1, 0});
    const bool k_blocked = block_interleave(k_len, k_str, A->type == TYPE_FLOAT ? 8 : 4);
    std::vector<int64_t> b_len = g.ABC.len;
    std::vector<std::vector<int64_t>> b_str = {g.ABC.stride[0], g.ABC.stride[1], g.ABC.stride[2]};
    append_modes(b_len, b_str, g.C_only, {-1, -1, 0});

    g.m = prod_len(g.AC.len);
    g.n = prod_len(g.BC.len);
    g.k = prod_len(k_len);
    g.batch = prod_len(b_len);
    const int64_t lim = (int64_t)1 << 31;
    if (g.m >= lim || g.n >= lim || g.k >= lim || g.batch >= lim) return TBLIS_STRA_ERR_TOO_LARGE;

    g.unit_rsA = first_stride(g.AC.len, g.AC.stride[0]);
    g.unit_rsC = first_stride(g.AC.len, g.AC.stride[1]);
    g.unit_csB = first_stride(g.BC.len, g.BC.stride[0]);
    g.unit_csC = first_stride(g.BC.len, g.BC.stride[1]);
    g.unit_ksA = first_stride(k_len, k_str[0], k_blocked ? 2 : 1);
    g.unit_ksB = first_stride(k_len, k_str[1], k_blocked ? 2 : 1);

    const std::vector<int64_t>* ml[9] = {&g.AC.len, &g.AC.len, &g.BC.len, &g.BC.len, &k_len, &k_len,
                                         &b_len, &b_len, &b_len};
    const std::vector<int64_t>* msd[9] = {&g.AC.stride[0], &g.AC.stride[1], &g.BC.stride[0], &g.BC.stride[1],
                                          &k_str[0], &k_str[1], &b_str[0], &b_str[1], &b_str[2]};
    for (int v = 0; v < 9; v++) { g.mode_len[v] = *ml[v]; g.mode_stride[v] = *msd[v]; }

    if (build_scatter)
    {
        scatter(g.AC.len, g.AC.stride[0], g.rsA);
        scatter(g.AC.len, g.AC.stride[1], g.rsC);
        scatter(g.BC.len, g.BC.stride[0], g.csB);
        scatter(g.BC.len, g.BC.stride[1], g.csC);
        scatter(k_len, k_str[0], g.ksA);
        scatter(k_len, k_str[1], g.ksB);
        scatter(b_len, b_str[0], g.bA);
        scatter(b_len, b_str[1], g.bB);
        scatter(b_len, b_str[2], g.bC);
    }
    return TBLIS_STRA_SUCCESS;
}

// ---- Strassen product tables ---------------------------------------------

namespace {

// Strassen 〈2,2,2〉: rows are sub-block ids 0..3 ((0,0),(0,1),(1,0),(1,1)),
// columns the 7 products; values from src/stra_internal/3t/strassen:1-14.
const int U[4][7] = {{1, 0, 1, 0, 1, -1, 0},
                     {0, 0, 0, 0, 1, 0, 1},
                     {0, 1, 0, 0, 0, 1, 0},
                     {1, 1, 0, 1, 0, 0, -1}};
const int V[4][7] = {{1, 1, 0, -1, 0, 1, 0},
                     {0, 0, 1, 0, 0, 1, 0},
                     {0, 0, 0, 1, 0, 0, 1},
                     {1, 0, -1, 0, 1, 0, 1}};
const int W[4][7] = {{1, 0, 0, 1, -1, 0, 1},
                     {0, 0, 1, 0, 1, 0, 0},
                     {0, 1, 0, 1, 0, 0, 0},
                     {1, -1, 1, 0, 0, 1, 0}};

FmmAlgorithm strassen_algorithm()
{
    FmmAlgorithm a;
    a.name = "strassen";
    a.mb = a.kb = a.nb = 2;
    a.rank = 7;
    for (int i = 0; i < 4; i++)
        for (int r = 0; r < 7; r++)
        {
            a.U.push_back(U[i][r]);
            a.V.push_back(V[i][r]);
            a.W.push_back(W[i][r]);
        }
    return a;
}

// The classical product of an mb x kb by kb x nb block grid: one product per
// (row, summed slice, column), each adding into one C block.
FmmAlgorithm classical_algorithm(int mb, int kb, int nb)
{
    FmmAlgorithm a;
    a.name = "classical" + std::to_string(mb) + std::to_string(kb) + std::to_string(nb);
    a.mb = mb; a.kb = kb; a.nb = nb;
    a.rank = mb * kb * nb;
    a.U.assign((size_t)(mb * kb * a.rank), 0);
    a.V.assign((size_t)(kb * nb * a.rank), 0);
    a.W.assign((size_t)(mb * nb * a.rank), 0);
    int r = 0;
    for (int i = 0; i < mb; i++)
        for (int t = 0; t < kb; t++)
            for (int j = 0; j < nb; j++, r++)
            {
                a.U[(size_t)((i * kb + t) * a.rank + r)] = 1;
                a.V[(size_t)((t * nb + j) * a.rank + r)] = 1;
                a.W[(size_t)((i * nb + j) * a.rank + r)] = 1;
            }
    return a;
}

// Strassen on the leading 2 x 2 x 2 blocks of a grid grown by one block along
// `axis` (0 rows of A and C, 1 the summed dimension, 2 columns of B and C),
// plus the classical products that the extra block needs: <3,2,2>, <2,3,2>
// and <2,2,3> with 7 + 4 = 11 products (against 12 classical).
FmmAlgorithm strassen_plus_classical(int axis)
{
    const FmmAlgorithm s = strassen_algorithm();
    FmmAlgorithm a;
    a.mb = axis == 0 ? 3 : 2; a.kb = axis == 1 ? 3 : 2; a.nb = axis == 2 ? 3 : 2;
    a.name = "strassen" + std::to_string(a.mb) + std::to_string(a.kb) + std::to_string(a.nb);
    a.rank = 11;
    a.U.assign((size_t)(a.mb * a.kb * 11), 0);
    a.V.assign((size_t)(a.kb * a.nb * 11), 0);
    a.W.assign((size_t)(a.mb * a.nb * 11), 0);
    for (int r = 0; r < 7; r++)
        for (int i = 0; i < 4; i++)
        {
            const int br = i / 2, bc = i % 2;
            a.U[(size_t)((br * a.kb + bc) * 11 + r)] = s.U[(size_t)(i * 7 + r)];
            a.V[(size_t)((br * a.nb + bc) * 11 + r)] = s.V[(size_t)(i * 7 + r)];
            a.W[(size_t)((br * a.nb + bc) * 11 + r)] = s.W[(size_t)(i * 7 + r)];
        }
    // the 4 classical products of the extra block row / slice / column
    int r = 7;
    for (int x = 0; x < 2; x++)
        for (int y = 0; y < 2; y++, r++)
        {
            int ai, aj, bi, bj, ci, cj;
            if (axis == 0)      { ai = 2; aj = x; bi = x; bj = y; ci = 2; cj = y; }   // C(2,y) += A(2,x) B(x,y)
            else if (axis == 1) { ai = x; aj = 2; bi = 2; bj = y; ci = x; cj = y; }   // C(x,y) += A(x,2) B(2,y)
            else                { ai = x; aj = y; bi = y; bj = 2; ci = x; cj = 2; }   // C(x,2) += A(x,y) B(y,2)
            a.U[(size_t)((ai * a.kb + aj) * 11 + r)] = 1;
            a.V[(size_t)((bi * a.nb + bj) * 11 + r)] = 1;
            a.W[(size_t)((ci * a.nb + cj) * 11 + r)] = 1;
        }
    return a;
}

// Exactness of an algorithm: sum_r U[A(i,t)][r] V[B(t',j)][r] W[C(i',j')][r]
// is 1 when t = t', i = i', j = j' and 0 otherwise (the matrix product).
bool algorithm_exact(const FmmAlgorithm& a)
{
    const int R = a.rank;
    if (a.mb < 1 || a.kb < 1 || a.nb < 1 || R < 1) return false;
    if (a.U.size() != (size_t)(a.mb * a.kb * R) || a.V.size() != (size_t)(a.kb * a.nb * R) ||
        a.W.size() != (size_t)(a.mb * a.nb * R))
        return false;
    for (int ia = 0; ia < a.mb * a.kb; ia++)
        for (int ib = 0; ib < a.kb * a.nb; ib++)
            for (int ic = 0; ic < a.mb * a.nb; ic++)
            {
                long long sum = 0;
                for (int r = 0; r < R; r++)
                    sum += (long long)a.U[(size_t)(ia * R + r)] * a.V[(size_t)(ib * R + r)] * a.W[(size_t)(ic * R + r)];
                const bool want = (ia % a.kb == ib / a.nb) && (ia / a.kb == ic / a.nb) && (ib % a.nb == ic % a.nb);
                if (sum != (want ? 1 : 0)) return false;
            }
    return true;
}

// Level-L table of an algorithm: product p has digits p_0 .. p_{L-1} (outer
// level most significant); a block of the Hm x Hk (A), Hk x Hn (B) and
// Hm x Hn (C) grids has row = sum_l row_l * base^(L-1-l), so for Strassen
// the 4 x 4 ids 4*row+col match src/stra_internal/3t/stra_mult_2level.cxx:341-353.
// False when a sum or a C update has more than 4 blocks.
bool build_table(const FmmAlgorithm& alg, int level, int id, ProductTable& t)
{
    t = ProductTable();
    t.level = level;
    t.algorithm = id;
    t.H = t.Hk = t.Hn = 1;
    for (int l = 0; l < level; l++) { t.H *= alg.mb; t.Hk *= alg.kb; t.Hn *= alg.nb; }
    if (level == 0)
    {
        Product p;
        p.na = p.nb = p.nc = 1;
        p.a[0] = {0, 0, 1}; p.b[0] = {0, 0, 1}; p.c[0] = {0, 0, 1};
        p.c_first[0] = 1;
        t.prod.push_back(p);
        return true;
    }
    int np = 1;
    for (int l = 0; l < level; l++) np *= alg.rank;
    for (int p = 0; p < np; p++)
    {
        std::vector<int> digits((size_t)level);
        int rem = p;
        for (int l = level - 1; l >= 0; l--) { digits[(size_t)l] = rem % alg.rank; rem /= alg.rank; }
        Product pr;
        auto expand = [&](const std::vector<int>& Mx, int rows, int cols, Term* out, int8_t& count) {
            struct Acc { int r, c, s; };
            std::vector<Acc> cur = {{0, 0, 1}};
            for (int l = 0; l < level; l++)
            {
                std::vector<Acc> nxt;
                for (auto& a : cur)
                    for (int id2 = 0; id2 < rows * cols; id2++)
                    {
                        const int v = Mx[(size_t)(id2 * alg.rank + digits[(size_t)l])];
                        if (!v) continue;
                        nxt.push_back({a.r * rows + id2 / cols, a.c * cols + id2 % cols, a.s * v});
                    }
                cur = nxt;
            }
            if (cur.size() > 4) return false;
            for (auto& a : cur)
                if (a.s != 1 && a.s != -1) return false;
            count = (int8_t)cur.size();
            for (size_t i = 0; i < cur.size(); i++)
                out[i] = {(int8_t)cur[i].r, (int8_t)cur[i].c, (int8_t)cur[i].s};
            return true;
        };
        if (!expand(alg.U, alg.mb, alg.kb, pr.a, pr.na) || !expand(alg.V, alg.kb, alg.nb, pr.b, pr.nb) ||
            !expand(alg.W, alg.mb, alg.nb, pr.c, pr.nc))
            return false;
        if (pr.na == 0 || pr.nb == 0 || pr.nc == 0) continue;   // a product that contributes nothing
        t.prod.push_back(pr);
    }
    // Mark the first product touching each C block (beta applied there once).
    std::vector<int> seen((size_t)(t.H * t.Hn), 0);
    for (auto& pr : t.prod)
        for (int i = 0; i < pr.nc; i++)
        {
            const int id2 = pr.c[i].r * t.Hn + pr.c[i].c;
            pr.c_first[i] = seen[(size_t)id2] ? 0 : 1;
            seen[(size_t)id2] = 1;
        }
    // every C block must be touched, or beta would not reach it
    for (int v : seen)
        if (!v) return false;
    return true;
}

struct Registry
{
    std::mutex mu;
    std::vector<FmmAlgorithm> algs;
    // tables per (algorithm, level 1..2); null where the kernels cannot run it
    std::vector<std::unique_ptr<ProductTable>> tab[3];
    Registry()
    {
        add(strassen_algorithm());
        add(classical_algorithm(2, 2, 2));
        add(strassen_plus_classical(0));
        add(strassen_plus_classical(1));
        add(strassen_plus_classical(2));
    }
    int add(const FmmAlgorithm& a)
    {
        const int id = (int)algs.size();
        algs.push_back(a);
        for (int level = 1; level <= 2; level++)
        {
            auto t = std::make_unique<ProductTable>();
            const bool ok = build_table(a, level, id, *t) && t->H <= 4 && t->Hk <= 4 && t->Hn <= 4 &&
                            !t->prod.empty() && t->prod.size() <= 49;
            tab[level].push_back(ok ? std::move(t) : nullptr);
        }
        return id;
    }
};

Registry& registry()
{
    static Registry r;
    return r;
}

thread_local int t_fmm = 0;

}  // namespace

int register_algorithm(const FmmAlgorithm& a)
{
    if (!algorithm_exact(a)) return -TBLIS_STRA_ERR_ARG;
    Registry& r = registry();
    std::lock_guard<std::mutex> lk(r.mu);
    if (r.algs.size() >= 64) return -TBLIS_STRA_ERR_TOO_LARGE;
    const int id = r.add(a);
    if (!r.tab[1][(size_t)id])
    {
        // keep the id (ids never move) but the kernels cannot run it
        return -TBLIS_STRA_ERR_UNSUPPORTED;
    }
    return id;
}

const FmmAlgorithm* algorithm_by_id(int id)
{
    Registry& r = registry();
    std::lock_guard<std::mutex> lk(r.mu);
    if (id < 0 || id >= (int)r.algs.size()) return nullptr;
    return &r.algs[(size_t)id];
}

const ProductTable* fmm_table(int id, int level)
{
    if (level == 0) return &strassen_table(0);
    if (level < 1 || level > 2) return nullptr;
    Registry& r = registry();
    std::lock_guard<std::mutex> lk(r.mu);
    if (id < 0 || id >= (int)r.algs.size()) return nullptr;
    return r.tab[level][(size_t)id].get();
}

void set_thread_algorithm(int id) { t_fmm = id; }
int thread_algorithm() { return t_fmm; }

const ProductTable& strassen_table(int level)
{
    struct Tables
    {
        ProductTable t[3];
        Tables()
        {
            const FmmAlgorithm s = strassen_algorithm();
            for (int l = 0; l < 3; l++) build_table(s, l, 0, t[l]);
        }
    };
    static const Tables tables;
    return tables.t[level < 0 ? 0 : level > 2 ? 2 : level];
}

const ProductTable& product_table(int level)
{
    if (level >= 1 && t_fmm != 0)
        if (const ProductTable* t = fmm_table(t_fmm, level)) return *t;
    return strassen_table(level);
}

namespace {

// Factored sums of one group from the coefficient matrix M (U for A, V for B).
PackGroup make_group(int level, const int (*M)[7], int group)
{
    PackGroup pg;
    if (level == 1)
    {
        pg.nt = 1;
        pg.t_s[0] = 1;
        for (int h = 0; h < 2; h++) { pg.row[0][h] = (int8_t)h; pg.col[0][h] = (int8_t)h; }
    }
    else
    {
        for (int id = 0; id < 4; id++)
        {
            if (!M[id][group]) continue;
            const int t = pg.nt++;
            pg.t_s[t] = (int8_t)M[id][group];
            for (int h = 0; h < 2; h++)
            {
                pg.row[t][h] = (int8_t)(2 * (id / 2) + h);
                pg.col[t][h] = (int8_t)(2 * (id % 2) + h);
            }
        }
    }
    for (int q = 0; q < 7; q++)
        for (int id = 0; id < 4; id++)
            if (M[id][q])
            {
                const int i = pg.o_n[q]++;
                pg.o_j[q][i] = (int8_t)id;
                pg.o_s[q][i] = (int8_t)M[id][q];
            }
    return pg;
}

// Expand a group's sums and compare them with the product table's terms.
bool group_matches(const PackGroup& pg, int level, int operand, int group)
{
    const ProductTable& t = strassen_table(level);
    for (int q = 0; q < 7; q++)
    {
        const Product& pr = t.prod[(size_t)(group * 7 + q)];
        const Term* want = operand == 0 ? pr.a : pr.b;
        const int nwant = operand == 0 ? pr.na : pr.nb;
        std::vector<std::tuple<int, int, int>> got, exp;
        for (int i = 0; i < pg.o_n[q]; i++)
        {
            const int j = pg.o_j[q][i];
            for (int c = 0; c < pg.nt; c++)
                got.emplace_back(pg.row[c][j / 2], pg.col[c][j % 2], pg.t_s[c] * pg.o_s[q][i]);
        }
        for (int i = 0; i < nwant; i++) exp.emplace_back(want[i].r, want[i].c, want[i].sign);
        std::sort(got.begin(), got.end());
        std::sort(exp.begin(), exp.end());
        if (got != exp) return false;
    }
    return true;
}

}  // namespace

const PackGroup* pack_group(int level, int operand, int group)
{
    struct Groups
    {
        std::vector<PackGroup> g[3][2];
        bool ok[3] = {false, false, false};
        Groups()
        {
            for (int level = 1; level <= 2; level++)
            {
                const int ngroups = level == 1 ? 1 : 7;
                ok[level] = true;
                for (int op = 0; op < 2; op++)
                    for (int G = 0; G < ngroups; G++)
                    {
                        g[level][op].push_back(make_group(level, op == 0 ? U : V, G));
                        ok[level] = ok[level] && group_matches(g[level][op].back(), level, op, G);
                    }
            }
        }
    };
    static const Groups groups;
    if (level < 1 || level > 2 || !groups.ok[level] || operand < 0 || operand > 1) return nullptr;
    if (thread_algorithm() != 0) return nullptr;   // the factored sums are Strassen's
    if (group < 0 || group >= (int)groups.g[level][operand].size()) return nullptr;
    return &groups.g[level][operand][(size_t)group];
}

}  // namespace tsb
