/* Test infrastructure only: the oracle. Nothing in the product links this.
 *
 * CPU restatement of the reference's hot-path arithmetic (see fg_oracle.h).
 * Every function cites the reference lines whose behaviour it restates; paths
 * are relative to the reference repository (AnonymousJune/flashgemm).
 *
 * Pinned against the reference itself: tests/test_oracle.py runs this file
 * and the reference compiled from its own sources (oracle/_ref, built by
 * oracle/Makefile) on the same seeded inputs, and against the committed golden
 * vectors in tests/golden/ that the compiled reference produced. */
#include "fg_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- scalar conversions ------------------------------------------------ */

/* Round-to-nearest-even FP32 -> BF16, the conversion vcvtne2ps2bf16 performs
 * between BF16 chain stages (multigemm/src/kernel_bf16.h:357-391). NaN stays a
 * quiet NaN. */
uint16_t orc_f32_to_bf16_rne(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40);
    uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return (uint16_t)(u >> 16);
}

/* Truncating FP32 -> BF16, the conversion the reference's test utilities use to
 * make BF16 inputs (multigemm/src/utils.h:20-33). */
uint16_t orc_f32_to_bf16_trunc(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    return (uint16_t)(u >> 16);
}

/* multigemm/src/utils.h:5-18 */
float orc_bf16_to_f32(uint16_t h)
{
    uint32_t u = (uint32_t)h << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

/* Signed saturation int32 -> int8 with no scale: vpmovsdb between INT8 chain
 * stages (multigemm/src/kernel_int8.h:329-385). */
int8_t orc_sat_s8(int32_t v)
{
    return (int8_t)(v > 127 ? 127 : (v < -128 ? -128 : v));
}

/* Column-strip width per thread: multigemm/src/flashgemm.c:40-52 (identical in
 * all three chain entry points). Panels of 32 columns start at each strip's
 * origin id*nb, so the strip width decides where the permutation's panels lie. */
long orc_strip_width(long N, int threads)
{
    long units = (N + 15) / 16;
    if (threads < 1) threads = 1;
    if (units % threads == 0) return (units / threads) * 16;
    return ((units + threads - 1) / threads) * 16;
}

/* ---- FP32 single GEMM -------------------------------------------------- */

/* C = A*B in FP64 from FP32 inputs: the non-reference accuracy oracle. */
void orc_sgemm_f64(const float *A, const float *B, double *C, long M, long N, long K)
{
#pragma omp parallel for schedule(static)
    for (long i = 0; i < M; ++i) {
        double *c = C + i * N;
        for (long j = 0; j < N; ++j) c[j] = 0.0;
        for (long k = 0; k < K; ++k) {
            double a = A[i * K + k];
            const float *b = B + k * N;
            for (long j = 0; j < N; ++j) c[j] += a * (double)b[j];
        }
    }
}

/* C = A*B in FP32 with one fused multiply-add per k in increasing k, the
 * arithmetic of the reference's vfmadd231ps register tiles
 * (singlegemm/src/kernel.h:8, multigemm/src/kernel_f32.h:3). With kblock > 0,
 * K is cut into blocks of kblock; each block is summed from zero and then added
 * into C, as singlegemm does with GEMM_K = 2048 (singlegemm/src/NN_mp.h:13) and
 * its ADD_C step (singlegemm/src/kernel.h:384-400). kblock = 0: one block. */
void orc_sgemm_f32(const float *A, const float *B, float *C, long M, long N, long K,
                   long kblock)
{
    if (kblock <= 0 || kblock > K) kblock = K > 0 ? K : 1;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < M; ++i) {
        float *c = C + i * N;
        float *part = (float *)malloc(sizeof(float) * (N > 0 ? N : 1));
        for (long j = 0; j < N; ++j) c[j] = 0.f;
        for (long k0 = 0; k0 < K; k0 += kblock) {
            long k1 = k0 + kblock < K ? k0 + kblock : K;
            for (long j = 0; j < N; ++j) part[j] = 0.f;
            for (long k = k0; k < k1; ++k) {
                float a = A[i * K + k];
                const float *b = B + k * N;
                for (long j = 0; j < N; ++j) part[j] = fmaf(a, b[j], part[j]);
            }
            if (k0 == 0)
                for (long j = 0; j < N; ++j) c[j] = part[j];
            else
                for (long j = 0; j < N; ++j) c[j] = c[j] + part[j];
        }
        free(part);
    }
}

/* ---- FP32 chain: multigemm/src/flashgemm.c:24-156 ------------------------ */

/* The reference's FP32 chain stores each stage's raw FP32 panel and reads it
 * back with the same layout (kernel_f32.h:470), so it is the mathematical chain
 * computed stage by stage in FP32 FMA. */
void orc_chain_f32(float *C, const float *B, long N, int n, const float *const *A,
                   const long *M, const long *K)
{
    const float *x = B;
    float *buf = NULL;
    for (int i = 0; i < n; ++i) {
        float *y = (i == n - 1) ? C : (float *)malloc(sizeof(float) * M[i] * N);
        orc_sgemm_f32(A[i], x, y, M[i], N, K[i], 0);
        free(buf);
        buf = (i == n - 1) ? NULL : y;
        x = y;
    }
    free(buf);
}

void orc_chain_f64(double *C, const float *B, long N, int n, const float *const *A,
                   const long *M, const long *K)
{
    double *x = (double *)malloc(sizeof(double) * K[0] * N);
    for (long t = 0; t < K[0] * N; ++t) x[t] = B[t];
    for (int i = 0; i < n; ++i) {
        double *y = (i == n - 1) ? C : (double *)malloc(sizeof(double) * M[i] * N);
#pragma omp parallel for schedule(static)
        for (long m = 0; m < M[i]; ++m) {
            double *c = y + m * N;
            for (long j = 0; j < N; ++j) c[j] = 0.0;
            for (long k = 0; k < K[i]; ++k) {
                double a = A[i][m * K[i] + k];
                const double *b = x + k * N;
                for (long j = 0; j < N; ++j) c[j] += a * b[j];
            }
        }
        free(x);
        x = (i == n - 1) ? NULL : y;
    }
    free(x);
}

/* ---- inter-stage panel permutation -------------------------------------- */

/* Between chain stages the reference stores a stage's narrowed output panel
 * P (M x w, w = 32 columns starting at a panel origin) row-major into the next
 * stage's packed-B buffer (kernel_bf16.h:356-391, kernel_int8.h:329-385), and
 * the next stage reads that buffer as packed B, whose layout interleaves
 * `g` consecutive k (g = 2 for BF16, kernel_bf16.h:6-32; g = 4 for INT8,
 * kernel_int8.h:6-50). Reading row-major data through the interleaved layout
 * permutes each g x 32 block:  X[g*q + r][j] = P[g*q + (g*j + r) / 32][(g*j + r) % 32].
 * `elt` is the element size in bytes. Panels narrower than 32 columns (the
 * reference's edge kernels, flashgemm.c:138-146) are left unpermuted. */
static void permute_panels(void *dst, const void *src, long rows, long N, int g, int elt,
                           int threads)
{
    const unsigned char *s = (const unsigned char *)src;
    unsigned char *d = (unsigned char *)dst;
    memcpy(d, s, (size_t)rows * N * elt);
    long nb = orc_strip_width(N, threads);
    for (long strip = 0; strip < N; strip += nb) {
        long se = strip + nb < N ? strip + nb : N;
        for (long p = strip; p + 32 <= se; p += 32) {
            for (long q = 0; q + g <= rows; q += g) {
                for (int r = 0; r < g; ++r)
                    for (int j = 0; j < 32; ++j) {
                        int t = g * j + r;
                        long srow = q + t / 32, scol = p + t % 32;
                        memcpy(d + ((q + r) * N + p + j) * elt, s + (srow * N + scol) * elt,
                               elt);
                    }
            }
        }
    }
}

/* ---- BF16 chain: multigemm/src/flashgemm.c:158-290 ----------------------- */

/* Stage products as vdpbf16ps computes them (kernel_bf16.h:37): per k pair,
 * the odd product then the even product are added into an FP32 accumulator
 * (each product of two BF16 values is exact in FP32). Between stages the FP32
 * result is rounded to BF16 (RNE) and, in REF mode, permuted per 2x32 block. */
int orc_chain_bf16(float *C, const uint16_t *B, long N, int n, const uint16_t *const *A,
                   const long *M, const long *K, int mode, int threads)
{
    for (int i = 0; i < n; ++i)
        if (K[i] % 2 != 0 || (i > 0 && K[i] != M[i - 1])) return -1;
    uint16_t *x = (uint16_t *)malloc(sizeof(uint16_t) * K[0] * N);
    memcpy(x, B, sizeof(uint16_t) * K[0] * N);
    for (int i = 0; i < n; ++i) {
        long Mi = M[i], Ki = K[i];
        float *acc = (i == n - 1) ? C : (float *)malloc(sizeof(float) * Mi * N);
#pragma omp parallel for schedule(static)
        for (long m = 0; m < Mi; ++m) {
            float *c = acc + m * N;
            for (long j = 0; j < N; ++j) c[j] = 0.f;
            for (long k = 0; k + 1 < Ki; k += 2) {
                float a0 = orc_bf16_to_f32(A[i][m * Ki + k]);
                float a1 = orc_bf16_to_f32(A[i][m * Ki + k + 1]);
                const uint16_t *b0 = x + k * N, *b1 = x + (k + 1) * N;
                for (long j = 0; j < N; ++j) {
                    float t = c[j] + a1 * orc_bf16_to_f32(b1[j]);
                    c[j] = t + a0 * orc_bf16_to_f32(b0[j]);
                }
            }
        }
        free(x);
        x = NULL;
        if (i < n - 1) {
            uint16_t *p = (uint16_t *)malloc(sizeof(uint16_t) * Mi * N);
            for (long t = 0; t < Mi * N; ++t) p[t] = orc_f32_to_bf16_rne(acc[t]);
            free(acc);
            x = (uint16_t *)malloc(sizeof(uint16_t) * Mi * N);
            if (mode == FG_ORC_REF)
                permute_panels(x, p, Mi, N, 2, 2, threads);
            else
                memcpy(x, p, sizeof(uint16_t) * Mi * N);
            free(p);
        }
    }
    free(x);
    return 0;
}

/* ---- INT8 chain: multigemm/src/flashgemm.c:292-424 ----------------------- */

/* Stage products as vpdpbusd computes them (kernel_int8.h:56): the weight byte
 * is read UNSIGNED and the activation byte SIGNED, four products summed into a
 * wrapping int32. Between stages: signed saturation to int8 with no scale
 * (kernel_int8.h:329-385) and, in REF mode, the 4x32 block permutation.
 *
 * REF mode also restates two tail behaviours of the reference's row blocking
 * (12-row blocks, then an 8-row and a 4-row block, kernel_int8.h:771-1057):
 *  - rows 12*floor(M/12) <= m < 4*floor(M/4) load the next packed-B k-quad
 *    before advancing the pointer (kernel_int8.h:405 vs :427, :590 vs :608),
 *    so weight quad s meets activation quad max(s-1, 0);
 *  - rows m >= 4*floor(M/4) are never written (kernel_int8.h:943-945): C keeps
 *    its previous contents there, and an intermediate's rows there are
 *    undefined (this restatement leaves them zero). */
int orc_chain_int8(int32_t *C, const uint8_t *B, long N, int n, const int8_t *const *A,
                   const long *M, const long *K, int mode, int threads)
{
    for (int i = 0; i < n; ++i)
        if (K[i] % 4 != 0 || (i > 0 && K[i] != M[i - 1])) return -1;
    int8_t *x = (int8_t *)malloc((size_t)K[0] * N);
    memcpy(x, B, (size_t)K[0] * N);
    for (int i = 0; i < n; ++i) {
        long Mi = M[i], Ki = K[i];
        long m_written = (mode == FG_ORC_REF) ? (Mi / 4) * 4 : Mi;
        long m_tail = (mode == FG_ORC_REF) ? (Mi / 12) * 12 : Mi;
        int32_t *acc = (int32_t *)malloc(sizeof(int32_t) * Mi * N);
        memset(acc, 0, sizeof(int32_t) * Mi * N);
#pragma omp parallel for schedule(static)
        for (long m = 0; m < m_written; ++m) {
            int64_t *c = (int64_t *)calloc((size_t)N, sizeof(int64_t));
            const uint8_t *a = (const uint8_t *)A[i] + m * Ki;
            for (long k = 0; k < Ki; ++k) {
                long kb = k;
                if (m >= m_tail) {
                    long s = k / 4;
                    kb = (s > 0 ? s - 1 : 0) * 4 + k % 4;
                }
                int32_t av = a[k];
                const int8_t *b = x + kb * N;
                for (long j = 0; j < N; ++j) c[j] += (int64_t)av * b[j];
            }
            for (long j = 0; j < N; ++j) acc[m * N + j] = (int32_t)(uint32_t)c[j];
            free(c);
        }
        free(x);
        x = NULL;
        if (i == n - 1) {
            memcpy(C, acc, sizeof(int32_t) * m_written * N);
        } else {
            int8_t *p = (int8_t *)malloc((size_t)Mi * N);
            for (long t = 0; t < Mi * N; ++t) p[t] = orc_sat_s8(acc[t]);
            x = (int8_t *)malloc((size_t)Mi * N);
            if (mode == FG_ORC_REF)
                permute_panels(x, p, Mi, N, 4, 1, threads);
            else
                memcpy(x, p, (size_t)Mi * N);
            free(p);
        }
        free(acc);
    }
    free(x);
    return 0;
}

double orc_rel_frob(const float *x, const double *ref, long count)
{
    double num = 0.0, den = 0.0;
    for (long t = 0; t < count; ++t) {
        double d = (double)x[t] - ref[t];
        num += d * d;
        den += ref[t] * ref[t];
    }
    return den > 0 ? sqrt(num / den) : sqrt(num);
}
