/*
 * The C caller shown in INTEGRATION.md, as a program the tests compile and
 * link against the library (-ltblis_stra_b200) with nothing but the public
 * header: a drop-in call of the reference's entry points on HOST buffers.
 *
 *   C(a,b,c,d) = alpha * A(e,f,a,c) * B(f,b,d,e) + beta * C(a,b,c,d)
 *
 * column-major, every extent E, entries from a fixed integer pattern the test
 * re-creates on its side.  Usage: capi_example LEVEL IMPL OUT_FILE [E]; writes
 * C (E^4 doubles, column-major) to OUT_FILE and exits with the status of the
 * call (0 = success; the TBLIS_STRA_* code otherwise).
 */
#include <stdio.h>
#include <stdlib.h>

#include "tblis_stra_b200.h"

static double pattern(long i, long mul, long add)
{
    return (double)((i * mul + add) % 2001 - 1000) / 1000.0;
}

int main(int argc, char** argv)
{
    if (argc < 4) { fprintf(stderr, "usage: %s LEVEL IMPL OUT_FILE [E]\n", argv[0]); return 64; }
    const int level = atoi(argv[1]);
    const int impl = atoi(argv[2]);
    const long E = argc > 4 ? atol(argv[4]) : 12;
    const long n = E * E * E * E;

    double* A = malloc(n * sizeof(double));
    double* B = malloc(n * sizeof(double));
    double* C = malloc(n * sizeof(double));
    if (!A || !B || !C) return 65;
    for (long i = 0; i < n; i++)
    {
        A[i] = pattern(i, 7919, 13);
        B[i] = pattern(i, 104729, 7);
        C[i] = pattern(i, 1299709, 3);
    }

    len_type len[4] = {E, E, E, E};
    stride_type st[4] = {1, E, E * E, E * E * E};      /* column-major, in elements */
    tblis_tensor tA = {TYPE_DOUBLE, 0, {0}, A, 4, len, st};
    tblis_tensor tB = {TYPE_DOUBLE, 0, {0}, B, 4, len, st};
    tblis_tensor tC = {TYPE_DOUBLE, 0, {0}, C, 4, len, st};
    *(double*)tA.scalar = 1.5;                         /* alpha = 1.5 * 1 */
    *(double*)tB.scalar = 1.0;
    *(double*)tC.scalar = 0.5;                         /* beta = 0.5 */

    if (tblis_stra_set_impl(impl) != TBLIS_STRA_SUCCESS) return 66;
    if (level == 0)      tblis_tensor_mult(NULL, NULL, &tA, "efac", &tB, "fbde", &tC, "abcd");
    else if (level == 1) stra_tblis_tensor_mult(NULL, NULL, &tA, "efac", &tB, "fbde", &tC, "abcd");
    else                 stra_tblis_tensor_mult_2level(NULL, NULL, &tA, "efac", &tB, "fbde", &tC, "abcd");
    const int status = tblis_stra_last_status();
    if (status != TBLIS_STRA_SUCCESS)
    {
        fprintf(stderr, "status %d: %s\n", status, tblis_stra_status_string(status));
        return status;
    }
    if (*(double*)tC.scalar != 1.0) return 67;         /* the call resets C's scalar to 1 */

    FILE* f = fopen(argv[3], "wb");
    if (!f || fwrite(C, sizeof(double), n, f) != (size_t)n) return 68;
    fclose(f);
    free(A); free(B); free(C);
    return 0;
}
