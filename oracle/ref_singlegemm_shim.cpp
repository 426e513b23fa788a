// Test infrastructure only: the oracle. Nothing in the product links this file.
//
// Builds the reference's own singlegemm implementation from its sources where
// they lie: singlegemm/FP32_ID23.c (the LibShalom_sgemm_mp dispatch at :35-62)
// and the headers it includes (NN_mp.h, set_TmTn.h, kernels, packing). The
// benchmark main() is renamed away, and the OpenBLAS check it links against is
// replaced by the stub cblas.h beside this file. Exported under ref_* names.

#define main ref_singlegemm_bench_main_unused
#define LibShalom_sgemm_mp ref_LibShalom_sgemm_mp
#include "singlegemm/FP32_ID23.c"
#undef main

extern "C" {

// FP32_ID23.c:35 with NUM = 24 compiled in; requires ref_set_thread_nums(24) first.
void ref_sgemm_mp(int transa, int transb, float *C, float *A, float *B, long M, long N, long K)
{
    ref_LibShalom_sgemm_mp(transa, transb, C, A, B, M, N, K);
}

// set_TmTn.h:61. Appends the divisors of num to a global list; call once per process.
void ref_set_thread_nums(int num) { LibShalom_set_thread_nums(num); }

// Same, after clearing the list: lets one process switch thread counts.
void ref_reset_thread_nums(int num)
{
    vec.clear();
    LibShalom_set_thread_nums(num);
}

// set_TmTn.h:10; returns the Tm x Tn grid it chose.
void ref_dete_grad_n(int T, long M, long N, int *tm, int *tn)
{
    Dete_grad_N_threads_nums(T, M, N, 0, 0);
    *tm = Tm;
    *tn = Tn;
}

// NN_mp.h:11 and :245, with an explicit thread count and grid.
void ref_sgemm_ngm(float *C, float *A, float *B, long M, long N, long K, int num, int tm, int tn)
{
    Small_NGM_NN_SGEMM(C, A, B, M, N, K, num, tm, tn);
}

void ref_sgemm_mgn(float *C, float *A, float *B, long M, long N, long K, int num, int tm, int tn)
{
    Small_MGN_NN_SGEMM(C, A, B, M, N, K, num, tm, tn);
}

}  // extern "C"
