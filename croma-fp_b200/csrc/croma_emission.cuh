// croma_emission.cuh -- device integrals of the per-snapshot emission
// (src/fp_shared_core.c:2008-2243, src/Synchrotron.c:62-103,
// src/EMISSION.c:297-308): the kernels shared by the reference-ABI entry
// points (ref_abi.cu) and the resident emission of a context (emission.cu).
// Internal header; the kernels are static, so every translation unit that
// includes it has its own copy.
#pragma once

#include "croma_segment.cuh"

namespace croma {

// The synchrotron prefactor A = sqrt(3) e^3 B / (2 m_e c^2) / (4 pi) of
// SYN_emissivity_from_arrays (src/Synchrotron.c:76) and
// prepare_synch_emission_cell_major (src/fp_shared_core.c:2093), split as
// a0 * B / den1 / den2 in the reference's evaluation order.
struct SynchPrefactor {
    double a0, den1, den2;
};
inline SynchPrefactor synch_prefactor()
{
    return SynchPrefactor{sqrt(3.0) * pow(4.8e-10, 3.0), 2.0 * 9.11e-28 * kC * kC, 4.0 * kPi};
}

// Q_one (src/EMISSION.c:297-308) times E n_gas, one thread per (cell, bin).
static __global__ void hadronic_emission_kernel(int ncell, int nbins, const double *crp, const double *n_gas,
                                         const double *beta_p, const double *dp, const double *kern,
                                         const double *E, double *out)
{
    const int ng = blockIdx.y * blockDim.y + threadIdx.y;
    const int icell = blockIdx.x * blockDim.x + threadIdx.x;
    if (icell >= ncell || ng >= nbins) return;
    const double *N = crp + (size_t)icell * NB;
    const double *f = kern + (size_t)ng * NB;
    double fpre = beta_p[0] * N[0] * f[0], integral = 0.0;
    for (int i = 1; i < NB; i++) {
        const double fn = beta_p[i] * N[i] * f[i];
        integral += (fpre + fn) * dp[i];
        fpre = fn;
    }
    out[(size_t)icell * nbins + ng] = E[ng] * (integral * 0.5) * n_gas[icell];
}

// prepare_ic_emission_cell_major (src/fp_shared_core.c:2131-2157): per
// (cell, band) the sum over electron bins of fic x N x dp, in bin order.
static __global__ void ic_emission_kernel(int ncell, int nbins, const double *cre, const double *fic,
                                   const double *dp, double *out)
{
    const int nic = blockIdx.y * blockDim.y + threadIdx.y;
    const int icell = blockIdx.x * blockDim.x + threadIdx.x;
    if (icell >= ncell || nic >= nbins) return;
    const double *N = cre + (size_t)icell * NB;
    const double *f = fic + (size_t)nic * NB;
    double integral = 0.0;
    for (int je = 0; je < NB; je++) integral += f[je] * N[je] * dp[je];
    out[(size_t)icell * nbins + nic] = integral;
}

// prepare_synch_emission_cell_major, pitch-kernel-table branch
// (src/fp_shared_core.c:2070-2112 with tracer_fp_interp_synch_kernel_logk :2054-2068).
static __global__ void synch_table_kernel(int ncell, int nfreq, int nlogb, double logb_min, double inv_dlogb,
                                   double a0, double den1, double den2, const double *table,
                                   const double *b_dyn, const double *logb, const double *cre,
                                   const double *dp, double *out)
{
    const int nf = blockIdx.y * blockDim.y + threadIdx.y;
    const int icell = blockIdx.x * blockDim.x + threadIdx.x;
    if (icell >= ncell || nf >= nfreq) return;
    const double *N = cre + (size_t)icell * NB;
    const double A = a0 * b_dyn[icell] / den1 / den2;
    const double u = (logb[icell] - logb_min) * inv_dlogb;
    int ib = (int)floor(u);
    if (ib < 0) ib = 0;
    if (ib > nlogb - 2) ib = nlogb - 2;
    double t = u - (double)ib;
    if (t < 0.0) t = 0.0;
    if (t > 1.0) t = 1.0;
    const double *k0 = table + ((size_t)ib * nfreq + nf) * NB;
    const double *k1 = table + ((size_t)(ib + 1) * nfreq + nf) * NB;
    double integral = 0.0;
    for (int je = 2; je < NB - 1 && N[je + 1] > 0.0; je++) {
        const double a = k0[je], b = k1[je];
        double K;
        if (t <= 0.0) K = a;
        else if (t >= 1.0) K = b;
        else if (a > 0.0 && b > 0.0) K = exp((1.0 - t) * log(a) + t * log(b));
        else K = (1.0 - t) * a + t * b;
        integral += N[je] * K * dp[je];
    }
    out[(size_t)icell * nfreq + nf] = A * integral;
}

// The synchrotron F(x) of the log-tabulated kernel at logx: 0 above the
// table, 0 below its first cell, the last value past its last cell, else
// 10^(log-linear interpolation) -- the lookup of SYN_emissivity_from_arrays
// (src/Synchrotron.c:81-97) and prepare_synch_pitch_kernel_table
// (src/fp_shared_core.c:2027-2042).
struct SynchFx {
    int nx;
    double xmin, inv_dlogx, logx_last, fx_last;
    const double *logx_tab, *logfx_tab;
    __device__ double operator()(double logx) const
    {
        if (!(logx <= logx_last)) return 0.0;
        const int ix = (int)floor((logx - xmin) * inv_dlogx);
        if (ix < 0) return 0.0;
        if (ix >= nx - 1) return fx_last;
        const double frac = (logx - logx_tab[ix]) * inv_dlogx;
        return pow(10.0, logfx_tab[ix] + frac * (logfx_tab[ix + 1] - logfx_tab[ix]));
    }
};

// sum_k F(logy[nf][je][k] - logb) w_k, the pitch-angle integral of one
// (frequency, electron bin) at one log B
__device__ __forceinline__ double pitch_integral(const SynchFx &F, const double *logy_row, const double *w,
                                                 int ntheta, double logb)
{
    double s = 0.0;
    for (int k = 0; k < ntheta; k++) s += F(logy_row[k] - logb) * w[k];
    return s;
}

// prepare_synch_pitch_kernel_table (src/fp_shared_core.c:2008-2052): table
// [nlogb][nfreq][npe], one thread per entry.
static __global__ void synch_pitch_table_kernel(SynchFx F, int nfreq, int ntheta, int nlogb, double logb_min,
                                         double inv_dlogb, const double *logy, const double *w, double *table)
{
    const long long total = (long long)nlogb * nfreq * NB;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int je = (int)(i % NB);
        const long long r = i / NB;
        const int nf = (int)(r % nfreq), ib = (int)(r / nfreq);
        const double logb = logb_min + (double)ib / inv_dlogb;
        table[i] = pitch_integral(F, logy + ((size_t)nf * NB + je) * ntheta, w, ntheta, logb);
    }
}

// prepare_synch_emission_cell_major without a pitch-kernel table
// (src/fp_shared_core.c:2113-2120 -> SYN_emissivity_from_arrays,
// src/Synchrotron.c:62-103): one warp per (cell, frequency).  The bins run
// from 2 up to the first je whose N[je+1] is not positive (found by a
// ballot); lanes take strided bins and a shuffle tree sums them.
static __global__ void __launch_bounds__(128) synch_theta_kernel(SynchFx F, int ncell, int nfreq, int ntheta,
                                                          double a0, double den1, double den2,
                                                          const double *logy, const double *w,
                                                          const double *b_dyn, const double *logb,
                                                          const double *cre, const double *dp, double *out)
{
    const int lane = threadIdx.x & 31;
    const long long idx = (long long)blockIdx.x * 4 + (threadIdx.x >> 5);
    if (idx >= (long long)ncell * nfreq) return;
    const int icell = (int)(idx / nfreq), nf = (int)(idx % nfreq);
    const double *N = cre + (size_t)icell * NB;
    int stop = NB - 1;   // first je >= 2 with N[je+1] <= 0, else npe - 1
    for (int j0 = 2; j0 < NB - 1; j0 += 32) {
        const int je = j0 + lane;
        const unsigned hit = __ballot_sync(0xffffffffu, je < NB - 1 && !(N[je + 1] > 0.0));
        if (hit) {
            stop = j0 + __ffs(hit) - 1;
            break;
        }
    }
    const double lb = logb[icell];
    double s = 0.0;
    for (int je = 2 + lane; je < stop; je += 32)
        s += N[je] * pitch_integral(F, logy + ((size_t)nf * NB + je) * ntheta, w, ntheta, lb) * dp[je];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) out[idx] = a0 * b_dyn[icell] / den1 / den2 * s;
}

}  // namespace croma
