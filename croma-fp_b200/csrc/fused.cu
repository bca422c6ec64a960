// fused.cu -- the on-chip FP64 evolve: the segment matrices of a tracer
// chunk are built and factored by one kernel, and a second kernel runs every
// sub-step of every segment with the spectrum held in registers.
//
// Per chunk of tracers (sized to the workspace budget) and species:
//   0. seg_pre_kernel, one thread per (segment, tracer): the segment's
//      interpolated background and the scalars of its coefficients, once for
//      both species.
//   1. factor_kernel, persistent: each warp takes tracers from an atomic
//      counter and factors every (segment[, on/off set]) of each: the loss /
//      diffusion terms of every bin in lane-strided loops into the warp's
//      slice of shared memory, the Chang-Cooper face weights (at 512 bins in
//      registers, where the rows use them; below, lane-strided into shared
//      memory) (losses / Dpp / CC assembly of src/fp_shared_core.c:729-842,
//      1241-1317, 2358-2431 and src/Chang_Cooper.c:22-184); rows a, b, c in
//      registers -- lane l owns rows [l*R, (l+1)*R), R = nb/32 -- and the
//      Thomas pivots d_i = b_i - a_i c_{i-1}/d_{i-1}, a chain of Moebius maps
//      composed per lane as 2x2 matrices and combined by a warp scan, after
//      which each lane re-runs the exact recurrence on its rows from the
//      scanned incoming pivot.  It stores 1/d, a/d and c/d per row.
//      Nothing here depends on the evolving spectra (the eta cap aside, which
//      then runs the chunk one segment at a time), so every segment of the
//      snapshot is factored by one launch with full occupancy.
//   2. steps_kernel, one warp per tracer: for each segment it loads the
//      factored rows (and the segment's source), and runs each sub-step as
//      the two first-order linear recurrences of fp_thomas_solve_ws
//      (src/fp_shared_core.c:226-257), each an affine warp scan: a local pass
//      per lane, five shuffle levels, a second local pass (substep); at 512
//      bins radix-4 scans of three shuffle levels with the back pass run
//      while the forward scan is in flight (substep4).  The proton kernel
//      records the spectrum at each segment start for the secondaries.
//   3. secondary_kernel: the electron source of every segment from those
//      proton spectra (prepare_secondary_sources_cell_major,
//      src/fp_shared_core.c:1591-1672), a tiled [segments*tracers x nb] .
//      [nb x nb] product on the FP64 tensor cores, between the proton and
//      the electron steps.
//
// Shared-memory rows are stored at (m % R) * kPitch + m / R, so the blocked reads
// of step 1 (lane l, row l*R + r and its neighbours) hit 32 distinct banks.
// Divisions by grid quantities use reciprocals tabulated on the host; the
// results agree with the reference's divisions to an ulp per operation.
// Spectra are cell-major [tracer][nb] so that a warp's rows are contiguous.
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "croma_segment.cuh"

namespace croma {

namespace {

constexpr int kR = NB / 32;          // rows per lane
// Row pitch of the swizzled arrays: both access patterns of the factor
// kernel -- lane-strided (m = 32 k + lane) and lane-blocked (m = R lane + r)
// -- then touch 16 distinct 8-byte bank pairs per half warp.
constexpr int kPitch = 32 + 16 / kR;
constexpr int kSw = kPitch * kR;     // swizzled row-array length
// One warp per block in the steps kernels: a finished tracer's slot is
// refilled at once instead of when the slowest warp of its block ends.
constexpr int kWarps = 1;            // warps per block
constexpr unsigned kFull = 0xffffffffu;
constexpr int kFacDoubles = 3 * NB;  // 1/d, a/d, c/d of one system
// Face weights of the factor kernel: at nb = 512 computed in registers where
// the rows use them, so each warp's shared memory holds only B and C and one
// 12-warp block (at most 168 registers, 160 KB of shared memory) fills an SM
// instead of 9 warps; at nb <= 256, where registers and not shared memory
// bound the warps, computed lane-strided into shared memory (two 9-warp
// blocks per SM).
constexpr bool kFacesInRegs = (NB >= 512);
constexpr int kFacWarps = (NB <= 256 ? 9 : 12);

// Grid tables of one species staged in shared memory by the factor kernel.
// X0..X3: protons expE, cp_Ep, cp_inv2mpkin, cp_inv_betap2; electrons
// ce_inv_beta2, ce_logp and the shared IC rows of z_curr, z_next.  RF: the
// face factor dx / (g_j + g_j+1) of the filled Dpp form.
enum { TB_P, TB_P2, TB_CUT, TB_2P, TB_DXF, TB_RF, TB_X0, TB_X1, TB_X2, TB_X3,
       TB_X4,                      // protons sig_eff, in swizzled order (row loss term)
       TB_IDX, TB_IDXL, TB_IDXR,   // 1/dp, 1/(p[m]-p[m-1]), 1/(p[m+1]-p[m]) in swizzled order
       kTab };
constexpr int kTabStride = (NB > kSw ? NB : kSw);   // doubles per staged table

// Per-segment scalars of one (segment slot, tracer): what the factor kernels
// of both species need of the schedule's segment and of the background
// interpolated to it, computed once by seg_pre_kernel.
struct SegPre {
    double n_gas, kbt, inv_kbt, log_n, adiab, synch_coeff, coulomb_coeff;
    double dt, dt_over_tloss_pref, dtT_e, alpha, dpp_inv;
    int flags;               // bit 0 active, 1 windowed, 2 interpolated, 3 "on" Dpp filled
    int sl, el, steps;       // Dpp window within the segment, sub-steps
};
enum { kPreActive = 1, kPreWindowed = 2, kPreInterp = 4, kPreFill = 8 };

struct FusedParams {
    SnapArgs a;              // spectra and sources cell-major [tracer][nb]
    GridTables gt;
    ModelParams mp;
    int g0, g1;              // segment slots of this launch
    int t0, nt;              // tracer chunk [t0, t0 + nt)
    int sets;                // factor sets per segment: 1 (on) or 2 (on, off)
    // One caller-defined segment shared by every tracer (run_tracer_pipeline):
    // when set, ex replaces the per-tracer schedule.
    int explicit_seg;
    SegInfo ex;
    // IC rows: shared row (stride 0) or per tracer, momentum-major
    // [nb][ntracer] (stride = ntracer)
    int ic_stride;
    const double *eta_scale; // [ntracer] Dpp eta-cap scale of slot g0, or null (no cap)
    double *fac;             // [2 species][g1 - g0][sets][nt][3][nb]
    SegPre *pre;             // [g1 - g0][nt]
    unsigned *work;          // [2] next-tracer counters of the factor kernels (per species)
    double *np_seg;          // [g1 - g0][nt][nb] proton spectra at segment starts, or null
    double *inje;            // [g1 - g0][nt][nb] electron source per segment, or null
    const int *np_min_qe;    // [nb]
    // solver calibration (the autotuner): when cal_spec is set, the steps
    // kernel reads and writes the spectra rows of tracer tl at cal_spec + tl nb
    // instead of the resident ones and stops after cal_steps sub-steps
    double *cal_spec;
    int cal_steps;
};

__device__ __forceinline__ SegInfo segment_of(const FusedParams &P, int t, int slot)
{
    return P.explicit_seg ? P.ex : seg_info(P.a.sched, t, slot, P.a.dt_snap);
}

__device__ __forceinline__ double *fac_ptr(const FusedParams &P, int S, int gi, int set, int tl)
{
    return P.fac + ((((size_t)S * (P.g1 - P.g0) + gi) * P.sets + set) * P.nt + tl) * kFacDoubles;
}

// Which factor sets a segment needs: 0 = Dpp on, 1 = off (windowed segments).
// The window is clamped to the segment's sub-steps as the steps kernel runs it.
__device__ __forceinline__ bool needs_set(const SegInfo &g, int set)
{
    if (!g.windowed) return set == 0;
    const int sl = min(max(g.sl, 0), g.steps), el = min(max(g.el, sl), g.steps);
    return (set == 0) ? el > sl : (sl > 0 || el < g.steps);
}

__device__ __forceinline__ int swz(int m) { return (m % kR) * kPitch + m / kR; }
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
__device__ __forceinline__ double sup(double v, int d) { return __shfl_up_sync(kFull, v, d); }
__device__ __forceinline__ double sdn(double v, int d) { return __shfl_down_sync(kFull, v, d); }
// 32-byte accesses of four consecutive doubles (sm_100 256-bit vector
// loads and stores).  The lanes of a warp own 128-byte row blocks, so a
// 16-byte access per lane would touch 32 sectors and use half of each (a
// scalar access a quarter); 32 bytes per lane use every sector fully.  The
// asm is volatile so that the per-step path's re-reads stay in its loop.
// ld4_cg / st4_cg: L2 only (rows and sources); ld4 / st4: the default caching.
__device__ __forceinline__ void ld4_cg(const double *p, double *v)
{
    asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(p));
}
__device__ __forceinline__ void ld4(const double *p, double *v)
{
    asm volatile("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(p) : "memory");
}
__device__ __forceinline__ void st4(double *p, const double *v)
{
    asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v[0]), "d"(v[1]), "d"(v[2]), "d"(v[3])
                 : "memory");
}
// st4 bypassing L1 (rows written for another kernel).
__device__ __forceinline__ void st4_cg(double *p, const double *v)
{
    asm volatile("st.global.cg.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v[0]), "d"(v[1]), "d"(v[2]), "d"(v[3])
                 : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int n = valid ? 16 : 0;   // 0 source bytes: the 16 destination bytes are zero-filled
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}

// Exact power-of-two rescaling of a 2x2 matrix (projective maps are
// unchanged by a common factor).
__device__ __forceinline__ void rescale2(double &m00, double &m01, double &m10, double &m11)
{
    const double mx = fmax(fmax(fabs(m00), fabs(m01)), fmax(fabs(m10), fabs(m11)));
    const long long ex = (__double_as_longlong(mx) >> 52) & 0x7ff;
    if (ex <= 0 || ex >= 2046) return;
    const double sc = __longlong_as_double((2046LL - ex) << 52);
    m00 *= sc; m01 *= sc; m10 *= sc; m11 *= sc;
}

// coulomb_kernel_fast with its erf / exp branch out of line: the proton
// terms otherwise inline four copies of it, and the factor kernel's code
// outgrows the instruction cache.  Same arithmetic.
__device__ __noinline__ double coulomb_slow(double x)
{
    return 0.5 * sqrt(kPi) * erf(sqrt(x)) - sqrt(x) * exp_tab(-x);
}
__device__ __forceinline__ double coulomb_one(double x)
{
    return (x > 40.0) ? 0.5 * sqrt(kPi) : coulomb_slow(x);
}

// Per-tracer constants of species S for one segment.
template <int S>
struct SegTerms {
    const GridTables *gt;
    double n_gas, kbt, inv_kbt, log_n, adiab;
    double synch_coeff, coulomb_coeff;
    double dt, dt_over_tloss_pref;   // protons: dt / T = sig_eff * dt_over_tloss_pref
    double dtT_e;                    // electrons: dt / 1e100
    double dpp_inv, dpp_scale;
    int dpp_fill;
    const double *ric, *ric_next;   // already offset to this tracer
    int ric_stride;                 // bin stride of the IC row; 0: the shared row, staged
    double alpha;
    int interp;

    // B = radp - 2 Dpp / p and C = Dpp at bin j, from the grid tables staged
    // in shared memory (tab, kTab arrays of nb)
    __device__ __forceinline__ void at(const double *tab, int j, double &B, double &C) const
    {
        const double p = tab[TB_P * kTabStride + j];
        const double p2 = tab[TB_P2 * kTabStride + j];
        const double cut = tab[TB_CUT * kTabStride + j];
        double D;
        if (!dpp_fill) D = p2 * (1.0 / (4.0 * 1.0e+5));
        else if (S == 0) D = p2 * dpp_inv * tab[TB_X0 * kTabStride + j] * cut;
        else D = p2 * dpp_inv * cut;
        D *= dpp_scale;
        double radp;
        if (S == 0) {
            const double xp = tab[TB_X1 * kTabStride + j] * inv_kbt;
            const double xe = xp * (kMe / kMp);
            const double sum = coulomb_one(xe) + coulomb_one(xp) * (kMe / kMp);
            const double thermal = 1.0 - kbt * tab[TB_X2 * kTabStride + j];
            const double coul = (thermal < 0.0)
                ? 0.0
                : kGyr * kC / (kMp * kGeV) * sum * n_gas * tab[TB_X3 * kTabStride + j] * thermal * 3.5e-29;
            radp = coul + adiab * p;
        } else {
            double r0, r1;
            if (ric_stride == 0) {
                r0 = tab[TB_X2 * kTabStride + j];
                r1 = tab[TB_X3 * kTabStride + j];
            } else {
                r0 = ric[j * ric_stride];
                r1 = ric_next[j * ric_stride];
            }
            const double r = interp ? lerp(r0, r1, alpha) : r0;
            // log(p / n) as log p - log n: the per-bin logarithm is tabulated
            const double coulomb = coulomb_coeff * (1.0 + (tab[TB_X1 * kTabStride + j] - log_n) * (1.0 / 74.8)) *
                                   tab[TB_X0 * kTabStride + j];
            radp = synch_coeff * p2 + r + coulomb + adiab * p;
        }
        B = radp - tab[TB_2P * kTabStride + j] * D;
        C = D;
    }

    // dT = dt / tloss of row r of a lane's block (swizzled index r * kPitch + lane)
    __device__ __forceinline__ double row_dT(const double *tab, int r, int lane) const
    {
        if (S == 0) return tab[TB_X4 * kTabStride + r * kPitch + lane] * dt_over_tloss_pref;
        return dtT_e;
    }
};

template <int S>
__device__ __forceinline__ SegTerms<S> seg_terms(const GridTables &gt, const Bg &bg, int dis,
                                                 const SnapArgs &a, const SegInfo &g, int t,
                                                 int ic_stride)
{
    SegTerms<S> T;
    T.gt = &gt;
    T.n_gas = bg.n_gas;
    T.kbt = bg.kbt;
    T.inv_kbt = 1.0 / bg.kbt;
    T.log_n = log(bg.n_gas);
    T.adiab = 1.0 / 3.0 * (dis ? 0.0 : bg.divv);
    const double b_ratio = bg.b_field * 1.0e+6 / 3.2;
    T.synch_coeff = 4.8e-4 * b_ratio * b_ratio * 9.11e-28 * 3.0e+10 * 3.1536e+16;
    T.coulomb_coeff = 3.05e-29 * bg.n_gas * kC * kGyr / (kMe * kGeV);
    T.dt = g.dt;
    T.dt_over_tloss_pref = g.dt / (1.0 / (0.5 * kC * bg.n_gas) / kGyr);
    T.dtT_e = g.dt / 1.0e+100;
    T.ric = a.ic_curr + (ic_stride ? t : 0);
    T.ric_next = a.ic_next + (ic_stride ? t : 0);
    T.ric_stride = ic_stride;
    T.alpha = g.alpha;
    T.interp = g.nseg > 1;
    T.dpp_inv = 0.0;
    T.dpp_scale = 1.0;
    T.dpp_fill = 0;
    return T;
}

// SegTerms of species S from the precomputed scalars of the segment.
template <int S>
__device__ __forceinline__ SegTerms<S> seg_terms_pre(const GridTables &gt, const SegPre *__restrict__ p,
                                                     const SnapArgs &a, int t, int ic_stride)
{
    SegTerms<S> T;
    T.gt = &gt;
    T.n_gas = p->n_gas;
    T.kbt = p->kbt;
    T.inv_kbt = p->inv_kbt;
    T.log_n = p->log_n;
    T.adiab = p->adiab;
    T.synch_coeff = p->synch_coeff;
    T.coulomb_coeff = p->coulomb_coeff;
    T.dt = p->dt;
    T.dt_over_tloss_pref = p->dt_over_tloss_pref;
    T.dtT_e = p->dtT_e;
    T.ric = a.ic_curr + (ic_stride ? t : 0);
    T.ric_next = a.ic_next + (ic_stride ? t : 0);
    T.ric_stride = ic_stride;
    T.alpha = p->alpha;
    T.interp = (p->flags & kPreInterp) ? 1 : 0;
    T.dpp_inv = 0.0;
    T.dpp_scale = 1.0;
    T.dpp_fill = 0;
    return T;
}

struct WarpSmem {
    double B[kSw], C[kSw];
    double Wp[kFacesInRegs ? 1 : kSw], Wm[kFacesInRegs ? 1 : kSw];
};


// Terms, faces and the rows a, b, c of one system: lane l holds rows
// [l*R, (l+1)*R) in A, Bd, Cc.
template <int S>
__device__ unsigned build_rows(const SegTerms<S> &T, const double *tab, int lane, WarpSmem &sm,
                               double A[kR], double Bd[kR], double Cc[kR])
{
    const SpeciesTables &st = T.gt->s[S];
    const double *x = st.p;
    unsigned err = 0;

    // Swizzled positions: for j = 32 k + lane, swz(j) = swz(lane) + k * 32 / R
    // and swz(j + 1) = swz(lane + 1) + k * 32 / R; for row m = R lane + r of
    // the lane's block, swz(m) = r * pitch + lane.
    constexpr int kStep = 32 / kR;
    const int sb0 = swz(lane), sb1 = swz(lane + 1);

    // terms, lane-strided
#pragma unroll 2
    for (int k = 0; k < kR; k++) {
        const int j = k * 32 + lane;
        double B, C;
        T.at(tab, j, B, C);
        sm.B[sb0 + k * kStep] = B;
        sm.C[sb0 + k * kStep] = C;
    }
    __syncwarp();
    // Faces j (between bins j and j+1).  In registers (kFacesInRegs) where the
    // rows use them: lane l's rows m = l R + r need faces m - 1 and m, so the
    // lane evaluates faces l R - 1 .. l R + R - 1 (the first one its left
    // neighbour evaluates too); else lane-strided into shared memory.  The
    // drift / diffusion ratio
    // (B_j + B_j+1) / (C_j + C_j+1) * dx: with the filled Dpp form the C sum
    // is kappa times a grid factor, so the division becomes a product with the
    // tabulated dx / (g_j + g_j+1) and 1 / kappa (equal to a few ulp).  The
    // division form is taken only when a lane of the warp needs it (the vote
    // keeps it from being computed predicated on every face).  Faces -1 and
    // nb - 1 do not exist.
    const double inv_kappa = T.dpp_fill ? 1.0 / (T.dpp_inv * T.dpp_scale) : 0.0;
    auto face = [&](int j, int sj, int sj1, double &wp, double &wm) {
        wp = 0.0;
        wm = 0.0;
        const bool exists = j >= 0 && j <= NB - 2;
        const double cl = exists ? sm.C[sj] : 0.0;
        const bool live = exists && fabs(cl) > 1.0e-200;
        const double bsum = exists ? sm.B[sj] + sm.B[sj1] : 0.0;
        const double rf = exists ? tab[TB_RF * kTabStride + sj] * inv_kappa : 0.0;
        const bool divide = live && !(T.dpp_fill && isfinite(rf));
        double w = bsum * rf;
        if (__any_sync(kFull, divide)) {
            if (divide) w = bsum / (cl + sm.C[sj1]) * tab[TB_DXF * kTabStride + sj];
        }
        if (live) face_weights_fast(w, wp, wm);
    };

    if (!kFacesInRegs) {
        // faces lane-strided into shared memory (j = 32 k + lane); face nb - 1
        // does not exist: its position swz(nb) is a padding word, never read
#pragma unroll 2
        for (int k = 0; k < kR; k++) {
            const int j = k * 32 + lane;
            const int s0 = sb0 + k * kStep, s1 = sb1 + k * kStep;
            double wp = 0.0, wm = 0.0;
            const double cl = sm.C[s0];
            const bool live = (j <= NB - 2) && fabs(cl) > 1.0e-200;
            const double bsum = sm.B[s0] + sm.B[s1];
            const double rf = tab[TB_RF * kTabStride + j] * inv_kappa;
            const bool divide = live && !(T.dpp_fill && isfinite(rf));
            double w = bsum * rf;
            if (__any_sync(kFull, divide)) {
                if (divide) w = bsum / (cl + sm.C[s1]) * tab[TB_DXF * kTabStride + j];
            }
            if (live) face_weights_fast(w, wp, wm);
            sm.Wp[kFacesInRegs ? 0 : s0] = wp;
            sm.Wm[kFacesInRegs ? 0 : s0] = wm;
        }
        __syncwarp();
    }

    // rows a, b, c of this lane (cc_build_{left,interior,right}, Chang_Cooper.c:66-184)
    const int row0 = lane * kR;
    double wpm = 0.0, wmm = 0.0;   // face m - 1
    if (kFacesInRegs) face(row0 - 1, lane > 0 ? (kR - 1) * kPitch + lane - 1 : 0, lane, wpm, wmm);
#pragma unroll
    for (int r = 0; r < kR; r++) {
        const int m = row0 + r;
        const int sm_m = r * kPitch + lane;
        const int sm_p = r > 0 ? (r - 1) * kPitch + lane : (kR - 1) * kPitch + lane - 1;   // swz(m - 1), m >= 1
        const int sm_n = r < kR - 1 ? (r + 1) * kPitch + lane : lane + 1;                  // swz(m + 1)
        double wpc, wmc;   // face m
        if (kFacesInRegs) {
            face(m, sm_m, sm_n, wpc, wmc);
        } else {
            wpc = sm.Wp[kFacesInRegs ? 0 : sm_m];
            wmc = sm.Wm[kFacesInRegs ? 0 : sm_m];
            if (m > 0) {
                wpm = sm.Wp[kFacesInRegs ? 0 : sm_p];
                wmm = sm.Wm[kFacesInRegs ? 0 : sm_p];
            }
        }
        const double k = T.dt * tab[TB_IDX * kTabStride + r * kPitch + lane];
        const double Cm = sm.C[r * kPitch + lane], Bm = sm.B[r * kPitch + lane], Dm = T.row_dT(tab, r, lane);
        double av = 0.0, bv, cv = 0.0;
        if (m == 0) {
            const double nC = sm.C[sm_n], nB = sm.B[sm_n];
            if (fabs(Cm) > 1.0e-200) {
                const double cm12 = 0.5 * (Cm + nC) * tab[TB_IDXR * kTabStride + r * kPitch + lane];
                bv = 1.0 + k * (0.0 + cm12 * wmc) + Dm;
                cv = k * cm12 * wpc;
            } else {
                bv = 1.0 + k * 0.0 + Dm;
                cv = k * 1.0 * 0.5 * (Bm + nB);
            }
        } else {
            const double pC = sm.C[sm_p], pB = sm.B[sm_p];
            if (m == NB - 1) {
                if (fabs(Cm) > 1.0e-200) {
                    const double cm_12 = 0.5 * (Cm + pC) * tab[TB_IDXL * kTabStride + r * kPitch + lane];
                    av = k * cm_12 * wmm;
                    bv = 1.0 + k * (cm_12 * wpm) + Dm;
                    if (isnan(av)) err |= kErrCcNan;
                } else {
                    double dlt = 0.0;
                    if (fabs(pC) > 1.0e-200)
                        dlt = face_delta((pB + Bm) / (pC + Cm) * (x[m] - x[m - 1]));
                    av = -dlt * 0.5 * (Bm + pB) * k;
                    bv = 1.0 + k * (0.5 * (pB + Bm)) + Dm;
                }
            } else {
                const double nC = sm.C[sm_n], nB = sm.B[sm_n];
                if (fabs(Cm) > 1.0e-200) {
                    const double cm_12 = 0.5 * (Cm + pC) * tab[TB_IDXL * kTabStride + r * kPitch + lane];
                    const double cm12 = 0.5 * (Cm + nC) * tab[TB_IDXR * kTabStride + r * kPitch + lane];
                    av = k * cm_12 * wmm;
                    bv = 1.0 + k * (cm_12 * wpm + cm12 * wmc) + Dm;
                    cv = k * cm12 * wpc;
                } else {
                    // interior row below the diffusion floor: every delta the
                    // reference reads here is zero (Chang_Cooper.c:91-103)
                    bv = 1.0 + k * (0.5 * (Bm + pB)) + Dm;
                    cv = k * 1.0 * 0.5 * (Bm + nB);
                }
            }
        }
        wpm = wpc;
        wmm = wmc;
        A[r] = av;
        Bd[r] = bv;
        Cc[r] = cv;
    }
    __syncwarp();
    return err;
}

// Thomas pivots of the rows a, b, c held as build_rows leaves them, in place:
// Bd <- 1/d, A <- a/d, Cc <- c/d (0 on the last row), with
// d_i = b_i + a_i c'_{i-1}, c'_i = -c_i / d_i (fp_thomas_solve_ws,
// src/fp_shared_core.c:226-257).  The chain of Moebius maps d -> b - e/d is
// composed per lane as 2x2 matrices and combined by a warp scan, after which
// each lane re-runs the exact recurrence on its rows from the scanned
// incoming pivot.  The lane's own matrix is rescaled to a largest entry in
// [1, 2); the scan's products then stay below 2^63 over its five levels, so
// they are not rescaled (powers of two are exact either way: same pivots).
__device__ __forceinline__ unsigned pivot_rows(double A[kR], double Bd[kR], double Cc[kR], int lane)
{
    unsigned err = 0;
    const int row0 = lane * kR;
    const double c_in = sup(Cc[kR - 1], 1);   // c of the row before this lane's first
    double t00 = 1.0, t01 = 0.0, t10 = 0.0, t11 = 1.0;
#pragma unroll
    for (int r = 0; r < kR; r++) {
        const double cprev = (r > 0) ? Cc[r - 1] : (lane > 0 ? c_in : 0.0);
        const double e = A[r] * cprev;
        const double n00 = Bd[r] * t00 - e * t10;
        const double n01 = Bd[r] * t01 - e * t11;
        t10 = t00;
        t11 = t01;
        t00 = n00;
        t01 = n01;
        if ((r & 3) == 3) rescale2(t00, t01, t10, t11);
    }
    rescale2(t00, t01, t10, t11);
#pragma unroll
    for (int lv = 0; lv < 5; lv++) {
        const int off = 1 << lv;
        const double u00 = sup(t00, off), u01 = sup(t01, off), u10 = sup(t10, off), u11 = sup(t11, off);
        if (lane >= off) {
            const double n00 = t00 * u00 + t01 * u10, n01 = t00 * u01 + t01 * u11;
            const double n10 = t10 * u00 + t11 * u10, n11 = t10 * u01 + t11 * u11;
            t00 = n00; t01 = n01; t10 = n10; t11 = n11;
        }
    }
    double vp = sup(t00, 1), vq = sup(t10, 1);
    double cp_prev = (lane == 0) ? 0.0 : -c_in * vq * rcp_nr(vp);
#pragma unroll
    for (int r = 0; r < kR; r++) {
        const int m = row0 + r;
        const double den = Bd[r] + A[r] * cp_prev;
        if (fabs(den) <= 1.0e-300) err |= kErrSingular;
        const double inv = rcp_nr(den);
        const double cr = Cc[r];
        Bd[r] = inv;
        A[r] = A[r] * inv;
        Cc[r] = (m == NB - 1) ? 0.0 : cr * inv;
        cp_prev = -cr * inv;
    }
    (void)vp;
    return err;
}

// Three row arrays of a lane to out[0..3nb): R contiguous doubles per array
// per lane (32-byte stores), nb doubles per array per warp.
__device__ __forceinline__ void store_rows(double *out, int lane, const double X[kR], const double Y[kR],
                                           const double Z[kR])
{
    const int row0 = lane * kR;
#pragma unroll
    for (int r = 0; r < kR; r += 4) {
        st4_cg(out + row0 + r, X + r);
        st4_cg(out + NB + row0 + r, Y + r);
        st4_cg(out + 2 * NB + row0 + r, Z + r);
    }
}

// One system of species S to out: factored (1/d, a/d, c/d) for the steps
// kernel, or the raw rows (a, b, c) for the per-step path, which factors
// them again on every sub-step.
template <int S, bool ROWS>
__device__ unsigned factor_store(const SegTerms<S> &T, const double *tab, int lane, WarpSmem &sm,
                                 double *out)
{
    double A[kR], Bd[kR], Cc[kR];
    unsigned err = build_rows<S>(T, tab, lane, sm, A, Bd, Cc);
    if (ROWS) {
        store_rows(out, lane, A, Bd, Cc);
        return err;
    }
    err |= pivot_rows(A, Bd, Cc, lane);
    store_rows(out, lane, Bd, A, Cc);
    return err;
}


// Factor kernel, persistent: each block stages the species' grid tables in
// shared memory once, then each warp takes tracers strided by the grid and
// factors every segment (and on/off set) of each (ROWS: stores the raw rows).
template <int S, bool ROWS>
__global__ void __launch_bounds__(kFacWarps * 32, (NB <= 256 ? 2 : 1)) factor_kernel(FusedParams P)
{
    extern __shared__ double4 smem_raw[];
    double *tab = reinterpret_cast<double *>(smem_raw);
    WarpSmem *smem = reinterpret_cast<WarpSmem *>(tab + kTab * kTabStride);
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const SnapArgs &a = P.a;
    const SpeciesTables &st = P.gt.s[S];
    for (int i = threadIdx.x; i < NB; i += blockDim.x) {
        tab[TB_P * kTabStride + i] = st.p[i];
        tab[TB_P2 * kTabStride + i] = st.p2[i];
        tab[TB_CUT * kTabStride + i] = st.exp_cut[i];
        tab[TB_2P * kTabStride + i] = st.two_over_p[i];
        tab[TB_DXF * kTabStride + (kFacesInRegs ? swz(i) : i)] = st.dxf[i];
        tab[TB_RF * kTabStride + (kFacesInRegs ? swz(i) : i)] = st.face_rf[i];
        if (S == 0) {
            tab[TB_X0 * kTabStride + i] = st.expE[i];
            tab[TB_X1 * kTabStride + i] = P.gt.cp_Ep[i];
            tab[TB_X2 * kTabStride + i] = P.gt.cp_inv2mpkin[i];
            tab[TB_X3 * kTabStride + i] = P.gt.cp_inv_betap2[i];
            tab[TB_X4 * kTabStride + swz(i)] = P.gt.sig_eff[i];
        } else {
            tab[TB_X0 * kTabStride + i] = P.gt.ce_inv_beta2[i];
            tab[TB_X1 * kTabStride + i] = P.gt.ce_logp[i];
            tab[TB_X2 * kTabStride + i] = (P.ic_stride == 0) ? a.ic_curr[i] : 0.0;
            tab[TB_X3 * kTabStride + i] = (P.ic_stride == 0) ? a.ic_next[i] : 0.0;
            tab[TB_X4 * kTabStride + swz(i)] = 0.0;
        }
        tab[TB_IDX * kTabStride + swz(i)] = st.inv_dx[i];
        tab[TB_IDXL * kTabStride + swz(i)] = st.inv_dxl[i];
        tab[TB_IDXR * kTabStride + swz(i)] = st.inv_dxr[i];
    }
    __syncthreads();
    // a warp takes one tracer at a time and factors all its segments (and
    // on/off sets) from the segments' precomputed scalars; after its first
    // tracer it takes the next one not yet taken (a counter the host zeroes
    // before the launch), so no warp is left with a whole extra tracer at the end
    const int stride = gridDim.x * kFacWarps;
    const int nslot = P.g1 - P.g0;
    int tl = blockIdx.x * kFacWarps + w;
#pragma unroll 1
    while (tl < P.nt) {
        const int t = P.t0 + tl;
        WarpSmem &ws = smem[w];
        const double eta = (P.mp.dpp_model != kDppOff && P.eta_scale) ? P.eta_scale[t] : 1.0;
#pragma unroll 1
        for (int gi = 0; gi < nslot; gi++) {
            const SegPre *__restrict__ pre = P.pre + (size_t)gi * P.nt + tl;
            const int flags = pre->flags;
            if (!(flags & kPreActive)) break;
            SegInfo g{};
            g.windowed = (flags & kPreWindowed) ? 1 : 0;
            g.sl = pre->sl;
            g.el = pre->el;
            g.steps = pre->steps;
            if (needs_set(g, 1) && P.sets < 2) {   // checked on the host; never write past the sets
                if (lane == 0) atomicOr(a.err, kErrBadInput);
                continue;
            }
#pragma unroll 1
            for (int set = 0; set < P.sets; set++) {
                if (!needs_set(g, set)) continue;
                SegTerms<S> T = seg_terms_pre<S>(P.gt, pre, a, t, P.ic_stride);
                if (set == 0) {
                    T.dpp_fill = (flags & kPreFill) ? 1 : 0;
                    T.dpp_inv = pre->dpp_inv;
                    T.dpp_scale = eta;
                }
                const unsigned err = factor_store<S, ROWS>(T, tab, lane, ws, fac_ptr(P, S, gi, set, tl));
                if (err && lane == 0) atomicOr(a.err, err);
                __syncwarp();
            }
        }
        unsigned next = 0;
        if (lane == 0) next = atomicAdd(P.work + S, 1u);
        tl = stride + (int)__shfl_sync(kFull, next, 0);
    }
}

// The factored rows of one segment as a lane holds them for its sub-steps,
// with the warp-scan multipliers.  hk[lv] / qk[lv] are zero on the lanes a
// scan level does not combine, and lane 0's a/d of row 0 and lane 31's c/d of
// the last row are zero, so the scans need no lane predicates.
template <bool SRC>
struct Coef {
    double inv[kR];      // 1 / d_i
    double h[kR];        // a_i / d_i      (forward recurrence)
    double q[kR];        // c_i / d_i      (back substitution)
    double sd[SRC ? kR : 1];  // dt * source_i / d_i
    double hk[5], qk[5];
    // products of h over the lower and upper half of the lane's rows, and of
    // q likewise: the local passes run as two half-length chains
    double hlo, hhi, qlo, qhi;
};

// The lane's rows of three arrays at in[0..3nb) (64 contiguous bytes each).
__device__ __forceinline__ void load_rows(const double *in, int lane, double X[kR], double Y[kR], double Z[kR])
{
    const int row0 = lane * kR;
#pragma unroll
    for (int r = 0; r < kR; r += 4) {
        ld4_cg(in + row0 + r, X + r);
        ld4_cg(in + NB + row0 + r, Y + r);
        ld4_cg(in + 2 * NB + row0 + r, Z + r);
    }
}

template <bool SRC>
__device__ __forceinline__ void scan_multipliers(Coef<SRC> &F, int lane);

// The rest of Coef once inv, h, q hold the lane's factored rows: the source
// term and the scan multipliers.
template <bool SRC>
__device__ __forceinline__ void finish_coef(Coef<SRC> &F, const double *src, double dt, int lane)
{
    const int row0 = lane * kR;
    if (lane == 0) F.h[0] = 0.0;
    if (lane == 31) F.q[kR - 1] = 0.0;
    if (SRC) {
#pragma unroll
        for (int r = 0; r < kR; r += 4) {
            double v[4];
            ld4_cg(src + row0 + r, v);
#pragma unroll
            for (int i = 0; i < 4; i++) F.sd[r + i] = (dt * v[i]) * F.inv[r + i];
        }
    }
    scan_multipliers<SRC>(F, lane);
}

// The half-chain products (hlo, hhi, qlo, qhi) and the warp-scan
// multipliers (hk, qk) of the lane's h and q rows.
template <bool SRC>
__device__ __forceinline__ void scan_multipliers(Coef<SRC> &F, int lane)
{
    double hlo = 1.0, hhi = 1.0, qlo = 1.0, qhi = 1.0;
#pragma unroll
    for (int r = 0; r < kR / 2; r++) {
        hlo *= F.h[r];
        qlo *= F.q[r];
        hhi *= F.h[r + kR / 2];
        qhi *= F.q[r + kR / 2];
    }
    F.hlo = hlo;
    F.hhi = hhi;
    F.qlo = qlo;
    F.qhi = qhi;
    double H = hlo * hhi, Q = qlo * qhi;
#pragma unroll
    for (int lv = 0; lv < 5; lv++) {
        const int off = 1 << lv;
        F.hk[lv] = (lane >= off) ? H : 0.0;
        F.qk[lv] = (lane + off < 32) ? Q : 0.0;
        const double Hu = sup(H, off), Qd = sdn(Q, off);
        if (lane >= off) H *= Hu;
        if (lane + off < 32) Q *= Qd;
    }
}

template <bool SRC>
__device__ __forceinline__ void load_coef(Coef<SRC> &F, const double *fac, const double *src, double dt,
                                          int lane)
{
    load_rows(fac, lane, F.inv, F.h, F.q);
    finish_coef<SRC>(F, src, dt, lane);
}

// One implicit sub-step: N <- M^{-1} (N + dt src) with the factored M.
// A shuffle from a lane outside the warp returns the caller's own (finite)
// value, which the zero multipliers discard exactly.  Each local pass runs
// as two independent half-length chains joined by one multiply-add, and the
// second pass seeds its upper (lower) half from the scanned carry directly,
// so no dependent chain is longer than half the lane's rows plus one.
template <bool SRC>
__device__ __forceinline__ void substep(const Coef<SRC> &F, double N[kR])
{
    constexpr int H2 = kR / 2;
    // forward: z_i = y_i + h_i z_{i-1}, y = N / d + dt src / d
    double alo = 0.0, ahi = 0.0;
#pragma unroll
    for (int r = 0; r < H2; r++) {
        N[r] = SRC ? fma(N[r], F.inv[r], F.sd[r]) : N[r] * F.inv[r];
        N[r + H2] = SRC ? fma(N[r + H2], F.inv[r + H2], F.sd[r + H2]) : N[r + H2] * F.inv[r + H2];
        alo = fma(F.h[r], alo, N[r]);
        ahi = fma(F.h[r + H2], ahi, N[r + H2]);
    }
    double acc = fma(F.hhi, alo, ahi);
#pragma unroll
    for (int lv = 0; lv < 5; lv++) acc = fma(F.hk[lv], sup(acc, 1 << lv), acc);
    const double cin = sup(acc, 1);
    double plo = cin, phi = fma(F.hlo, cin, alo);
#pragma unroll
    for (int r = 0; r < H2; r++) {
        plo = fma(F.h[r], plo, N[r]);
        phi = fma(F.h[r + H2], phi, N[r + H2]);
        N[r] = plo;
        N[r + H2] = phi;
    }
    // back substitution: x_i = z_i + q_i x_{i+1}
    alo = 0.0;
    ahi = 0.0;
#pragma unroll
    for (int r = H2 - 1; r >= 0; r--) {
        alo = fma(F.q[r], alo, N[r]);
        ahi = fma(F.q[r + H2], ahi, N[r + H2]);
    }
    acc = fma(F.qlo, ahi, alo);
#pragma unroll
    for (int lv = 0; lv < 5; lv++) acc = fma(F.qk[lv], sdn(acc, 1 << lv), acc);
    const double cout = sdn(acc, 1);
    phi = cout;
    plo = fma(F.qhi, cout, ahi);
#pragma unroll
    for (int r = H2 - 1; r >= 0; r--) {
        phi = fma(F.q[r + H2], phi, N[r + H2]);
        plo = fma(F.q[r], plo, N[r]);
        N[r + H2] = phi;
        N[r] = plo;
    }
}

// The steps kernel's registers bound its occupancy: warps are spread over
// the SM's four sub-partitions, each with a quarter of the register file, so
// at 512 bins (16 rows a lane) 8 warps per SM allow 255 registers a thread
// and 12 allow 168, at 256 bins 16 allow 128 and 20 allow 102.  The
// kSolveScanShared variant keeps the per-segment constants that a sub-step
// only reads -- dt src / d of each row and the ten scan multipliers -- in the
// warp's slice of shared memory ([r][lane] and [level][lane], one
// conflict-free 8-byte read each per sub-step) instead of registers, for the
// larger warp count.  The kSolveScanRhs variant also moves 1 / d of each
// row there, as (1 / d, dt src / d) pairs ([r][lane], one conflict-free
// 16-byte read per row and sub-step): the lane then holds only N, h and q
// (about 100 registers at 512 bins), for 16 warps per SM at 512 bins and 24
// at 256 with one warp per block (12 and 20 with two).
constexpr int kCoefSmemDoubles = NB + 10 * 32;       // per warp: dt src / d, hk, qk
constexpr int kRhsSmemDoubles = 2 * NB + 10 * 32;    // per warp: (1 / d, dt src / d), hk, qk

// substep() with the per-segment constants of the warp's shared-memory slice
// wsm.  RHS false (kSolveScanShared): dt src / d at wsm[r * 32 + lane] (SRC),
// the scan multipliers at wsm[NB + lv * 32 + lane] (hk) and
// wsm[NB + (5 + lv) * 32 + lane] (qk).  RHS true (kSolveScanRhs): the pair
// (1 / d, dt src / d) of row r at double2 index r * 32 + lane, hk and qk
// after the 2 NB doubles of pairs.  Same arithmetic as substep().
template <bool SRC, bool RHS>
__device__ __forceinline__ void substep_sm(const Coef<SRC> &F, const double *wsm, int lane, double N[kR])
{
    constexpr int H2 = kR / 2;
    const double *sm = wsm + lane;
    const double2 *rhs = reinterpret_cast<const double2 *>(wsm) + lane;
    const double *hk = sm + (RHS ? 2 * NB : NB), *qk = hk + 5 * 32;
    double alo = 0.0, ahi = 0.0;
#pragma unroll
    for (int r = 0; r < H2; r++) {
        if (RHS) {
            const double2 u = rhs[r * 32], v = rhs[(r + H2) * 32];
            N[r] = SRC ? fma(N[r], u.x, u.y) : N[r] * u.x;
            N[r + H2] = SRC ? fma(N[r + H2], v.x, v.y) : N[r + H2] * v.x;
        } else {
            N[r] = SRC ? fma(N[r], F.inv[r], sm[r * 32]) : N[r] * F.inv[r];
            N[r + H2] = SRC ? fma(N[r + H2], F.inv[r + H2], sm[(r + H2) * 32]) : N[r + H2] * F.inv[r + H2];
        }
        alo = fma(F.h[r], alo, N[r]);
        ahi = fma(F.h[r + H2], ahi, N[r + H2]);
    }
    double acc = fma(F.hhi, alo, ahi);
#pragma unroll
    for (int lv = 0; lv < 5; lv++) acc = fma(hk[lv * 32], sup(acc, 1 << lv), acc);
    const double cin = sup(acc, 1);
    double plo = cin, phi = fma(F.hlo, cin, alo);
#pragma unroll
    for (int r = 0; r < H2; r++) {
        plo = fma(F.h[r], plo, N[r]);
        phi = fma(F.h[r + H2], phi, N[r + H2]);
        N[r] = plo;
        N[r + H2] = phi;
    }
    alo = 0.0;
    ahi = 0.0;
#pragma unroll
    for (int r = H2 - 1; r >= 0; r--) {
        alo = fma(F.q[r], alo, N[r]);
        ahi = fma(F.q[r + H2], ahi, N[r + H2]);
    }
    acc = fma(F.qlo, ahi, alo);
#pragma unroll
    for (int lv = 0; lv < 5; lv++) acc = fma(qk[lv * 32], sdn(acc, 1 << lv), acc);
    const double cout = sdn(acc, 1);
    phi = cout;
    plo = fma(F.qhi, cout, ahi);
#pragma unroll
    for (int r = H2 - 1; r >= 0; r--) {
        phi = fma(F.q[r + H2], phi, N[r + H2]);
        plo = fma(F.q[r], plo, N[r]);
        N[r + H2] = phi;
        N[r] = plo;
    }
}

// kSolveScanRhs's coefficient load: the (1 / d, dt src / d) pairs of the
// lane's rows go from the factored rows (and the source) straight to the
// warp's slice, h and q into registers, and the scan multipliers, formed as
// load_coef forms them, into the slice after the pairs.
template <bool SRC>
__device__ __forceinline__ void load_coef_rhs(Coef<SRC> &F, const double *fac, const double *src, double dt,
                                              int lane, double *wsm)
{
    const int row0 = lane * kR;
    double2 *rhs = reinterpret_cast<double2 *>(wsm) + lane;
    __syncwarp();   // the previous run's reads of the slice are done
#pragma unroll
    for (int r = 0; r < kR; r += 4) {
        double vi[4], vs[4] = {0.0, 0.0, 0.0, 0.0};
        ld4_cg(fac + row0 + r, vi);
        if (SRC) ld4_cg(src + row0 + r, vs);
#pragma unroll
        for (int i = 0; i < 4; i++) rhs[(r + i) * 32] = make_double2(vi[i], SRC ? (dt * vs[i]) * vi[i] : 0.0);
    }
#pragma unroll
    for (int r = 0; r < kR; r += 4) {
        ld4_cg(fac + NB + row0 + r, F.h + r);
        ld4_cg(fac + 2 * NB + row0 + r, F.q + r);
    }
    if (lane == 0) F.h[0] = 0.0;
    if (lane == 31) F.q[kR - 1] = 0.0;
    scan_multipliers<SRC>(F, lane);
    double *hk = wsm + 2 * NB + lane;
#pragma unroll
    for (int lv = 0; lv < 5; lv++) {
        hk[lv * 32] = F.hk[lv];
        hk[(5 + lv) * 32] = F.qk[lv];
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Short-chain sub-step (kSolveScan4).  substep() runs, per sub-step, the
// forward recurrence (local pass, 5-level warp scan, carry shuffle, second
// local pass) and then the back substitution the same way, one after the
// other: two scans of six dependent shuffles each plus four dependent local
// passes.  This form shortens that chain in two ways.
//
// * Radix-4 warp scans: the carry into lane i is gathered from the
//   aggregates of lanes i-1..i-4 (four shuffles issued together), then from
//   those partial carries at lanes i-4, i-8, i-12, then at i-16: three
//   dependent shuffle levels instead of six, exclusive directly.
// * The back substitution's local pass runs on the forward pass's raw
//   (zero-carry) values while the forward scan is in flight.  Both
//   recurrences are linear, so the true back aggregate of the lane is the raw
//   one plus per-segment constants times the forward carry; the forward
//   carry then reaches the rows as z = raw + (product of h) carry, a chain of
//   multiplies that runs while the back scan is in flight.
//
// The sums are the same as substep()'s, regrouped (results agree to
// rounding, not bit for bit).
struct Scan4 {
    double fw[3];    // forward level 1: weights of the aggregates of lanes i-2, i-3, i-4 (i-1: 1)
    double fp[4];    // forward levels 2, 3: products of H over lanes i-4..i-1, i-8.., i-12.., i-16..
    double bw[3];    // the same for the back substitution (lanes i+2, i+3, i+4)
    double bp[4];
    double kh;       // back aggregate of the upper half's carry response to z at its first row - 1
    double qk, kc;   // qlo kh, and the full back aggregate's response to the forward carry
};

// Forward exclusive scan: the carry into this lane (z at the last row of the
// lane below), from each lane's zero-carry aggregate a.  Weights outside the
// warp are zero, so the shuffles need no lane predicates (a shuffle from
// outside the warp returns the caller's own finite value).
__device__ __forceinline__ double scan4_up(double a, const double fw[3], const double fp[4], int lane)
{
    const double s1 = sup(a, 1), s2 = sup(a, 2), s3 = sup(a, 3), s4 = sup(a, 4);
    const double S = fma(fw[0], s2, lane >= 1 ? s1 : 0.0) + fma(fw[2], s4, fw[1] * s3);
    const double t4 = sup(S, 4), t8 = sup(S, 8), t12 = sup(S, 12);
    const double E = fma(fp[0], t4, S) + fma(fp[2], t12, fp[1] * t8);
    return fma(fp[3], sup(E, 16), E);
}

// Back exclusive scan: the carry into this lane from above (x at the first
// row of the lane above).
__device__ __forceinline__ double scan4_down(double a, const double bw[3], const double bp[4], int lane)
{
    const double s1 = sdn(a, 1), s2 = sdn(a, 2), s3 = sdn(a, 3), s4 = sdn(a, 4);
    const double S = fma(bw[0], s2, lane <= 30 ? s1 : 0.0) + fma(bw[2], s4, bw[1] * s3);
    const double t4 = sdn(S, 4), t8 = sdn(S, 8), t12 = sdn(S, 12);
    const double E = fma(bp[0], t4, S) + fma(bp[2], t12, bp[1] * t8);
    return fma(bp[3], sdn(E, 16), E);
}

// The Scan4 constants of the lane's coefficients (after load_coef).
template <bool SRC>
__device__ __forceinline__ void make_scan4(const Coef<SRC> &F, Scan4 &R, int lane)
{
    const double H = F.hlo * F.hhi, Q = F.qlo * F.qhi;   // products over the lane's rows
    {
        const double h1 = sup(H, 1), h2 = sup(H, 2), h3 = sup(H, 3), h4 = sup(H, 4);
        const double w3 = h1 * h2, w4 = w3 * h3, p4 = w4 * h4;
        const double p8 = p4 * sup(p4, 4);
        const double p12 = p8 * sup(p4, 8);
        const double p16 = p8 * sup(p8, 8);
        R.fw[0] = lane >= 2 ? h1 : 0.0;
        R.fw[1] = lane >= 3 ? w3 : 0.0;
        R.fw[2] = lane >= 4 ? w4 : 0.0;
        R.fp[0] = lane >= 4 ? p4 : 0.0;
        R.fp[1] = lane >= 8 ? p8 : 0.0;
        R.fp[2] = lane >= 12 ? p12 : 0.0;
        R.fp[3] = lane >= 16 ? p16 : 0.0;
    }
    {
        const double q1 = sdn(Q, 1), q2 = sdn(Q, 2), q3 = sdn(Q, 3), q4 = sdn(Q, 4);
        const double w3 = q1 * q2, w4 = w3 * q3, p4 = w4 * q4;
        const double p8 = p4 * sdn(p4, 4);
        const double p12 = p8 * sdn(p4, 8);
        const double p16 = p8 * sdn(p8, 8);
        R.bw[0] = lane <= 29 ? q1 : 0.0;
        R.bw[1] = lane <= 28 ? w3 : 0.0;
        R.bw[2] = lane <= 27 ? w4 : 0.0;
        R.bp[0] = lane <= 27 ? p4 : 0.0;
        R.bp[1] = lane <= 23 ? p8 : 0.0;
        R.bp[2] = lane <= 19 ? p12 : 0.0;
        R.bp[3] = lane <= 15 ? p16 : 0.0;
    }
    // the back aggregate of each half applied to the half's forward carry
    // response (the running products of h from the half's first row)
    constexpr int H2 = kR / 2;
    double clo[H2], chi[H2];
    double c0 = 1.0, c1 = 1.0;
#pragma unroll
    for (int r = 0; r < H2; r++) {
        c0 *= F.h[r];
        c1 *= F.h[r + H2];
        clo[r] = c0;
        chi[r] = c1;
    }
    double kl = 0.0, kh = 0.0;
#pragma unroll
    for (int r = H2 - 1; r >= 0; r--) {
        kl = fma(F.q[r], kl, clo[r]);
        kh = fma(F.q[r + H2], kh, chi[r]);
    }
    R.kh = kh;
    R.qk = F.qlo * kh;
    R.kc = fma(R.qk, F.hlo, kl);
}

template <bool SRC>
__device__ __forceinline__ void substep4(const Coef<SRC> &F, const Scan4 &R, int lane, double N[kR])
{
    constexpr int H2 = kR / 2;
    // forward, zero carry into each half: N <- the raw chain values
    double alo = 0.0, ahi = 0.0;
#pragma unroll
    for (int r = 0; r < H2; r++) {
        const double ylo = SRC ? fma(N[r], F.inv[r], F.sd[r]) : N[r] * F.inv[r];
        const double yhi = SRC ? fma(N[r + H2], F.inv[r + H2], F.sd[r + H2]) : N[r + H2] * F.inv[r + H2];
        alo = fma(F.h[r], alo, ylo);
        ahi = fma(F.h[r + H2], ahi, yhi);
        N[r] = alo;
        N[r + H2] = ahi;
    }
    const double af = fma(F.hhi, alo, ahi);
    // back aggregates of the raw values, independent of the forward scan
    double blo = 0.0, bhi = 0.0;
#pragma unroll
    for (int r = H2 - 1; r >= 0; r--) {
        blo = fma(F.q[r], blo, N[r]);
        bhi = fma(F.q[r + H2], bhi, N[r + H2]);
    }
    const double bpre = fma(R.qk, alo, fma(F.qlo, bhi, blo));
    const double cin = scan4_up(af, R.fw, R.fp, lane);
    const double zh = fma(F.hlo, cin, alo);          // z at the lower half's last row
    const double cout = scan4_down(fma(R.kc, cin, bpre), R.bw, R.bp, lane);
    const double bhi_t = fma(R.kh, zh, bhi);         // the upper half's true back aggregate
    // the forward carry's response: z = raw + (running product of h) carry
    double d = cin, e = zh;
#pragma unroll
    for (int r = 0; r < H2; r++) {
        d *= F.h[r];
        e *= F.h[r + H2];
        N[r] += d;
        N[r + H2] += e;
    }
    // back substitution: x_i = z_i + q_i x_{i+1}
    double phi = cout, plo = fma(F.qhi, cout, bhi_t);
#pragma unroll
    for (int r = H2 - 1; r >= 0; r--) {
        phi = fma(F.q[r + H2], phi, N[r + H2]);
        plo = fma(F.q[r], plo, N[r]);
        N[r + H2] = phi;
        N[r] = plo;
    }
}

// ---------------------------------------------------------------------------
// FP32-refined sub-step (the "precision" form of the chosen path): the solve
// of each sub-step in FP32 followed by one iterative-refinement sweep whose
// residual is formed in FP64, the result kept in FP64.
//
//   y   = N / d + dt src / d                       FP64 (the scaled right-hand side)
//   x0  = M^-1 y                                   FP32, the same two recurrences
//   rho = y - (u - h u_{-1}),  u = x0 - q x0_{+1}  FP64: r / d - M x0 / d with M = L U,
//                                                  L = (d, -a), U = (1, -c/d) the
//                                                  FP64 factors of the segment
//   e   = M^-1 rho                                 FP32
//   N   = x0 + e                                   FP64
//
// The FP32 solves see y scaled by a per-segment power of two s (exact), so
// that the largest |y| of the tracer is near 1 and the spectra, which span
// more decades than FP32 does, keep their dominant bins in range; rho is
// scaled by s 2^20.  The factored rows stay FP64 (the residual needs them);
// the multipliers of the FP32 recurrences are their FP32 roundings.
struct Coef32 {
    float h[kR], q[kR];
    float hk[5], qk[5];
    float hlo, hhi, qlo, qhi;
};

__device__ __forceinline__ float supf(float v, int d) { return __shfl_up_sync(kFull, v, d); }
__device__ __forceinline__ float sdnf(float v, int d) { return __shfl_down_sync(kFull, v, d); }

template <bool SRC>
__device__ __forceinline__ void make_coef32(const Coef<SRC> &F, Coef32 &G, int lane)
{
#pragma unroll
    for (int r = 0; r < kR; r++) {
        G.h[r] = (float)F.h[r];
        G.q[r] = (float)F.q[r];
    }
    float hlo = 1.0f, hhi = 1.0f, qlo = 1.0f, qhi = 1.0f;
#pragma unroll
    for (int r = 0; r < kR / 2; r++) {
        hlo *= G.h[r];
        qlo *= G.q[r];
        hhi *= G.h[r + kR / 2];
        qhi *= G.q[r + kR / 2];
    }
    G.hlo = hlo;
    G.hhi = hhi;
    G.qlo = qlo;
    G.qhi = qhi;
    float H = hlo * hhi, Q = qlo * qhi;
#pragma unroll
    for (int lv = 0; lv < 5; lv++) {
        const int off = 1 << lv;
        G.hk[lv] = (lane >= off) ? H : 0.0f;
        G.qk[lv] = (lane + off < 32) ? Q : 0.0f;
        const float Hu = supf(H, off), Qd = sdnf(Q, off);
        if (lane >= off) H *= Hu;
        if (lane + off < 32) Q *= Qd;
    }
}

// x <- M^-1 x in FP32, x holding the scaled right-hand side (substep's two
// recurrences without the 1/d and source step).
__device__ __forceinline__ void solve32(const Coef32 &G, float x[kR])
{
    constexpr int H2 = kR / 2;
    float alo = 0.0f, ahi = 0.0f;
#pragma unroll
    for (int r = 0; r < H2; r++) {
        alo = fmaf(G.h[r], alo, x[r]);
        ahi = fmaf(G.h[r + H2], ahi, x[r + H2]);
    }
    float acc = fmaf(G.hhi, alo, ahi);
#pragma unroll
    for (int lv = 0; lv < 5; lv++) acc = fmaf(G.hk[lv], supf(acc, 1 << lv), acc);
    const float cin = supf(acc, 1);
    float plo = cin, phi = fmaf(G.hlo, cin, alo);
#pragma unroll
    for (int r = 0; r < H2; r++) {
        plo = fmaf(G.h[r], plo, x[r]);
        phi = fmaf(G.h[r + H2], phi, x[r + H2]);
        x[r] = plo;
        x[r + H2] = phi;
    }
    alo = 0.0f;
    ahi = 0.0f;
#pragma unroll
    for (int r = H2 - 1; r >= 0; r--) {
        alo = fmaf(G.q[r], alo, x[r]);
        ahi = fmaf(G.q[r + H2], ahi, x[r + H2]);
    }
    acc = fmaf(G.qlo, ahi, alo);
#pragma unroll
    for (int lv = 0; lv < 5; lv++) acc = fmaf(G.qk[lv], sdnf(acc, 1 << lv), acc);
    const float cout = sdnf(acc, 1);
    phi = cout;
    plo = fmaf(G.qhi, cout, ahi);
#pragma unroll
    for (int r = H2 - 1; r >= 0; r--) {
        phi = fmaf(G.q[r + H2], phi, x[r + H2]);
        plo = fmaf(G.q[r], plo, x[r]);
        x[r + H2] = phi;
        x[r] = plo;
    }
}

// Power-of-two scale that brings the tracer's largest scaled right-hand side
// |N / d + dt src / d| near 1 (1 for an all-zero spectrum).
template <bool SRC>
__device__ __forceinline__ double refine_scale(const Coef<SRC> &F, const double N[kR])
{
    double m = 0.0;
#pragma unroll
    for (int r = 0; r < kR; r++) m = fmax(m, fabs(N[r] * F.inv[r]) + (SRC ? fabs(F.sd[r]) : 0.0));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(kFull, m, off));
    if (!(m > 0.0) || !isfinite(m)) return 1.0;
    int e = ilogb(m);
    e = max(-1000, min(1000, e));
    return ldexp(1.0, -e);
}

template <bool SRC>
__device__ __forceinline__ void substep_refined(const Coef<SRC> &F, const Coef32 &G, double N[kR], double s)
{
    const double inv_s = 1.0 / s, s2 = s * 1048576.0, inv_s2 = inv_s * (1.0 / 1048576.0);
    float x[kR], e[kR];
#pragma unroll
    for (int r = 0; r < kR; r++) {
        const double y = SRC ? fma(N[r], F.inv[r], F.sd[r]) : N[r] * F.inv[r];
        x[r] = (float)(y * s);
    }
    solve32(G, x);
    // u_r = x0_r - q_r x0_{r+1}; the row after the lane's last is the next
    // lane's first (the last lane's last q is zero, so its own value is harmless)
    const double xnext = sdn((double)x[0] * inv_s, 1);
    const double ulast = (double)x[kR - 1] * inv_s - F.q[kR - 1] * xnext;
    double uprev = sup(ulast, 1);   // lane 0: h of row 0 is zero
#pragma unroll
    for (int r = 0; r < kR; r++) {
        const double x0 = (double)x[r] * inv_s;
        const double x1 = (r < kR - 1) ? (double)x[r + 1] * inv_s : xnext;
        const double u = x0 - F.q[r] * x1;
        const double y = SRC ? fma(N[r], F.inv[r], F.sd[r]) : N[r] * F.inv[r];
        const double rho = (y - u) + F.h[r] * uprev;
        e[r] = (float)(rho * s2);
        uprev = u;
    }
    solve32(G, e);
#pragma unroll
    for (int r = 0; r < kR; r++) N[r] = (double)x[r] * inv_s + (double)e[r] * inv_s2;
}

// ---------------------------------------------------------------------------
// Warp PCR sub-step: parallel cyclic reduction of the tridiagonal system
// b_i x_i - a_i x_{i-1} - c_i x_{i+1} = N_i + dt src_i, the algorithm of the
// reference's solve_cc_pcr_kernel (src/fp_cuda_solver.cu:144-206) with one
// warp per system instead of one thread block: each lane keeps its R rows in
// registers, and at stride s every row combines with rows i - s and i + s
// read back from the warp's slice of shared memory (swizzled rows, so both
// partners of a lane's row r sit in distinct banks):
//   alpha = a_i / b_{i-s},  gamma = c_i / b_{i+s},
//   b <- b - alpha c_{i-s} - gamma a_{i+s},  a <- alpha a_{i-s},
//   c <- gamma c_{i+s},  d <- d + alpha d_{i-s} + gamma d_{i+s},
// log2(nb) levels, then x_i = d_i / b_i.  The rows a, b, c are rebuilt from
// the segment's factored rows (d = 1/inv, a = h d, c = q d,
// b = d + a q_{i-1}).  It does O(nb log nb) work and data movement per
// sub-step against the scan's O(nb); the autotuner times both.
struct PcrSmem {
    double a[kSw], b[kSw], c[kSw], d[kSw];
};

template <bool SRC>
__device__ __forceinline__ void pcr_rows_from_factored(Coef<SRC> &F, double cc[kR], int lane)
{
    // in place: inv -> b, h -> a, sd -> dt src; c into cc (q is read as the
    // previous row's multiplier, so it stays)
    const double q_in = sup(F.q[kR - 1], 1);   // q of the row before this lane's first
#pragma unroll
    for (int r = 0; r < kR; r++) {
        const double dd = 1.0 / F.inv[r];
        const double qprev = (r > 0) ? F.q[r - 1] : (lane > 0 ? q_in : 0.0);
        const double aa = F.h[r] * dd;
        cc[r] = F.q[r] * dd;
        F.inv[r] = dd + aa * qprev;
        if (SRC) F.sd[r] = F.sd[r] * dd;
        F.h[r] = aa;
    }
}

template <bool SRC>
__device__ __forceinline__ void substep_pcr(const Coef<SRC> &F, const double cc[kR], double N[kR], PcrSmem &sm,
                                            int lane)
{
    double a[kR], b[kR], c[kR];
#pragma unroll
    for (int r = 0; r < kR; r++) {
        a[r] = F.h[r];
        b[r] = F.inv[r];
        c[r] = cc[r];
        N[r] = SRC ? N[r] + F.sd[r] : N[r];
    }
#pragma unroll 1
    for (int st = 1; st < NB; st <<= 1) {
        __syncwarp();
#pragma unroll
        for (int r = 0; r < kR; r++) {
            const int o = r * kPitch + lane;
            sm.a[o] = a[r];
            sm.b[o] = b[r];
            sm.c[o] = c[r];
            sm.d[o] = N[r];
        }
        __syncwarp();
#pragma unroll
        for (int r = 0; r < kR; r++) {
            const int m = lane * kR + r;
            double na = 0.0, nb = b[r], nc = 0.0, nd = N[r];
            if (m - st >= 0) {
                const int o = swz(m - st);
                const double al = a[r] / sm.b[o];
                na = al * sm.a[o];
                nb -= al * sm.c[o];
                nd += al * sm.d[o];
            }
            if (m + st < NB) {
                const int o = swz(m + st);
                const double ga = c[r] / sm.b[o];
                nc = ga * sm.c[o];
                nb -= ga * sm.a[o];
                nd += ga * sm.d[o];
            }
            a[r] = na;
            b[r] = nb;
            c[r] = nc;
            N[r] = nd;
        }
    }
#pragma unroll
    for (int r = 0; r < kR; r++) N[r] = N[r] / b[r];
}

// Sub-step solvers of the steps kernel: the FP64 warp-scan Thomas (its
// per-segment constants in registers, or in shared memory to leave registers
// for more warps), the short-chain FP64 form (radix-4 scans, back pass
// overlapping the forward scan), the warp scan with FP32 solves refined by
// an FP64 residual, and warp PCR.
enum { kSolveScan = 0, kSolveRefined = 1, kSolvePcr = 2, kSolveScanShared = 3, kSolveScanRhs = 4,
       kSolveScan4 = 5 };

// Steps kernel: warp w of block b runs every segment [g0, g1) of tracer
// t0 + b * WPB + w for species S with sub-step solver SOLVER.
template <int S, bool SRC, int SOLVER, int WPB>
__global__ void __launch_bounds__(WPB * 32,
                                  (SOLVER == kSolveScanShared ? (NB <= 256 ? 20 : 12)
                                   : SOLVER == kSolveScanRhs  ? (WPB == 1 ? (NB <= 256 ? 24 : 16) : (NB <= 256 ? 20 : 12))
                                                              : (NB <= 256 ? 16 : 8)) / WPB)
    steps_kernel(FusedParams P)
{
    extern __shared__ double4 steps_smem[];
    constexpr bool kSm = SOLVER == kSolveScanShared;
    constexpr bool kRhs = SOLVER == kSolveScanRhs;
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int tl = blockIdx.x * WPB + w;
    if (tl >= P.nt) return;
    const int t = P.t0 + tl;
    const SnapArgs &a = P.a;
    const int row0 = lane * kR;
    double *Nrow = (P.cal_spec ? P.cal_spec + (size_t)tl * NB : (S == 0 ? a.crp : a.cre) + (size_t)t * NB) + row0;
    double N[kR];
#pragma unroll
    for (int r = 0; r < kR; r += 4) ld4(Nrow + r, N + r);
    const double *qsrc = (S == 0) ? a.qpi : a.qepri;
    Coef<SRC> F;
    Coef32 G;
    Scan4 R4;
    double cc[SOLVER == kSolvePcr ? kR : 1];
    PcrSmem *pcr_sm = reinterpret_cast<PcrSmem *>(steps_smem) + w;
    double *coef_sm = reinterpret_cast<double *>(steps_smem) + (size_t)w * (kRhs ? kRhsSmemDoubles : kCoefSmemDoubles);
    double scale = 1.0;
    int budget = P.cal_steps > 0 ? P.cal_steps : 0x7fffffff;
    const int nslot = P.g1 - P.g0;
#pragma unroll 1
    for (int gi = 0; gi < nslot && budget > 0; gi++) {
        const SegPre *__restrict__ pre = P.pre + (size_t)gi * P.nt + tl;
        const int flags = pre->flags;
        if (!(flags & kPreActive)) continue;
        SegInfo g{};
        g.windowed = (flags & kPreWindowed) ? 1 : 0;
        g.sl = pre->sl;
        g.el = pre->el;
        g.steps = pre->steps;
        g.dt = pre->dt;
        // the next segment's rows (Dpp-on set) and source into L2 while this
        // segment's sub-steps run: its loads then wait on L2, not on DRAM
        if (gi + 1 < nslot) {
            const double *nf = fac_ptr(P, S, gi + 1, 0, tl) + row0;
            if (lane < 2)   // and the next segment's scalars this loop reads (dt .. steps of its SegPre)
                prefetch_l2(reinterpret_cast<const char *>(P.pre + (size_t)(gi + 1) * P.nt + tl) +
                            (lane ? offsetof(SegPre, steps) : offsetof(SegPre, dt)));
            prefetch_l2(nf);
            prefetch_l2(nf + NB);
            prefetch_l2(nf + 2 * NB);
            if (SRC && S == 1 && P.inje) prefetch_l2(P.inje + ((size_t)(gi + 1) * P.nt + tl) * NB + row0);
        }
        if (S == 0 && P.np_seg && !P.cal_spec) {
            double *o = P.np_seg + ((size_t)gi * P.nt + tl) * NB + row0;
#pragma unroll
            for (int r = 0; r < kR; r += 4) st4_cg(o + r, N + r);
        }
        const double *src = nullptr;
        if (SRC) {
            src = (S == 1 && P.inje) ? P.inje + ((size_t)gi * P.nt + tl) * NB
                                     : qsrc + (size_t)t * NB;
        }
        // runs of sub-steps with one coefficient set: Dpp off before the
        // window, on inside it, off after it (all on when not windowed)
        const int sl = g.windowed ? min(max(g.sl, 0), g.steps) : 0;
        const int el = g.windowed ? min(max(g.el, sl), g.steps) : g.steps;
        int cur = -1;
#pragma unroll 1
        for (int k = 0; k < 3; k++) {
            const int want = (k == 1) ? 0 : 1;
            int run_n = (k == 0) ? sl : (k == 1 ? el - sl : g.steps - el);
            if (run_n <= 0) continue;
            if (want >= P.sets) {   // no off set in the workspace: report, leave N as it was
                if (lane == 0) atomicOr(a.err, kErrBadInput);
                return;
            }
            run_n = min(run_n, budget);
            budget -= run_n;
            if (want != cur) {
                if (kRhs) load_coef_rhs<SRC>(F, fac_ptr(P, S, gi, want, tl), src, g.dt, lane, coef_sm);
                else load_coef<SRC>(F, fac_ptr(P, S, gi, want, tl), src, g.dt, lane);
                if (SOLVER == kSolveRefined) make_coef32<SRC>(F, G, lane);
                if (SOLVER == kSolveScan4) make_scan4<SRC>(F, R4, lane);
                if (SOLVER == kSolvePcr) pcr_rows_from_factored<SRC>(F, cc, lane);
                if (kSm) {
                    __syncwarp();   // the previous run's reads of the slice are done
                    if (SRC) {
#pragma unroll
                        for (int r = 0; r < kR; r++) coef_sm[r * 32 + lane] = F.sd[r];
                    }
#pragma unroll
                    for (int lv = 0; lv < 5; lv++) {
                        coef_sm[NB + lv * 32 + lane] = F.hk[lv];
                        coef_sm[NB + (5 + lv) * 32 + lane] = F.qk[lv];
                    }
                    __syncwarp();
                }
                cur = want;
            }
            if (SOLVER == kSolveRefined) {
                scale = refine_scale<SRC>(F, N);
#pragma unroll 1
                for (int istep = 0; istep < run_n; istep++) substep_refined<SRC>(F, G, N, scale);
            } else if (SOLVER == kSolvePcr) {
#pragma unroll 1
                for (int istep = 0; istep < run_n; istep++) substep_pcr<SRC>(F, cc, N, *pcr_sm, lane);
            } else if (kSm) {
#pragma unroll 2
                for (int istep = 0; istep < run_n; istep++) substep_sm<SRC, false>(F, coef_sm, lane, N);
            } else if (kRhs) {
#pragma unroll 1
                for (int istep = 0; istep < run_n; istep++) substep_sm<SRC, true>(F, coef_sm, lane, N);
            } else if (SOLVER == kSolveScan4) {
#pragma unroll 2   // two sub-steps per trip, as for substep (no spills at 254 registers)
                for (int istep = 0; istep < run_n; istep++) substep4<SRC>(F, R4, lane, N);
            } else {
                // two sub-steps per trip: the carried spectrum keeps its
                // registers across the loop (fewer copies per sub-step)
#pragma unroll 2
                for (int istep = 0; istep < run_n; istep++) substep<SRC>(F, N);
            }
            if (budget <= 0) break;
        }
    }
#pragma unroll
    for (int r = 0; r < kR; r += 4) st4(Nrow + r, N + r);
}

// Per-step kernel (the plain path): warp w of block b advances tracer
// t0 + b * kWarps + w through the sub-steps of segment slot g0 with the
// reference's per-step data contract -- every sub-step reads the rows a, b, c
// of its on/off set, the source and N from memory, solves M N' = N + dt src
// with the pivots recomputed (tracer_fp_cpu_evolve, src/tracer_fp_cpu.c:149-190;
// fp_thomas_solve_ws, src/fp_shared_core.c:226-257) and writes N back.
template <int S, bool SRC>
__global__ void __launch_bounds__(kWarps * 32, (NB <= 256 ? 20 : 12)) plain_steps_kernel(FusedParams P)
{
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int tl = blockIdx.x * kWarps + w;
    if (tl >= P.nt) return;
    const int t = P.t0 + tl;
    const SnapArgs &a = P.a;
    const SegPre *__restrict__ pre = P.pre + tl;
    const int flags = pre->flags;
    if (!(flags & kPreActive)) return;
    const int windowed = (flags & kPreWindowed) ? 1 : 0;
    const int sl = pre->sl, el = pre->el, steps = pre->steps;
    const double dt = pre->dt;
    const int row0 = lane * kR;
    double *Nrow = (S == 0 ? a.crp : a.cre) + (size_t)t * NB + row0;
    const double *src = nullptr;
    if (SRC) src = (S == 1 && P.inje) ? P.inje + (size_t)tl * NB : ((S == 0) ? a.qpi : a.qepri) + (size_t)t * NB;
    Coef<SRC> F;
    double N[kR];
#pragma unroll 1
    for (int istep = 0; istep < steps; istep++) {
        const int set = (!windowed || (istep >= sl && istep < el)) ? 0 : 1;
        if (set >= P.sets) {   // no off set in the workspace: report, leave N as it is
            if (lane == 0) atomicOr(a.err, kErrBadInput);
            return;
        }
        // rows a, b, c of the set: A <- a, inv <- b, q <- c, then the pivots
        load_rows(fac_ptr(P, S, 0, set, tl), lane, F.h, F.inv, F.q);
#pragma unroll
        for (int r = 0; r < kR; r += 4) ld4(Nrow + r, N + r);
        const unsigned err = pivot_rows(F.h, F.inv, F.q, lane);
        if (__any_sync(kFull, err != 0)) {
            if (lane == 0) atomicOr(a.err, kErrSingular);
            return;
        }
        finish_coef<SRC>(F, src, dt, lane);
        substep<SRC>(F, N);
#pragma unroll
        for (int r = 0; r < kR; r += 4) st4(Nrow + r, N + r);
    }
}

// The per-segment scalars of every (slot, tracer) of the chunk, one thread
// each: the schedule's segment (tracer_fp_batch.c segment split), the
// background interpolated to it, the loss coefficients and the "on" Dpp form
// (prepare_momentumdiff_cell_major, src/fp_shared_core.c:1241-1317) -- the
// same arithmetic the factor kernels would repeat per species and set.
__global__ void __launch_bounds__(256) seg_pre_kernel(FusedParams P)
{
    const SnapArgs &a = P.a;
    const long long total = (long long)(P.g1 - P.g0) * P.nt;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int gi = (int)(i / P.nt);
        const int tl = (int)(i - (long long)gi * P.nt);
        const int t = P.t0 + tl;
        SegPre o{};
        const SegInfo g = segment_of(P, t, P.g0 + gi);
        if (g.active) {
            const Bg bg = load_bg(a, t, g);
            const int dis = a.dis ? a.dis[t] : 0;
            const SegTerms<0> T = seg_terms<0>(P.gt, bg, dis, a, g, t, P.ic_stride);
            const DppForm on = dpp_form(P.mp, P.mp.dpp_model, bg, segment_tacc(P.mp, a, g));
            o.n_gas = T.n_gas;
            o.kbt = T.kbt;
            o.inv_kbt = T.inv_kbt;
            o.log_n = T.log_n;
            o.adiab = T.adiab;
            o.synch_coeff = T.synch_coeff;
            o.coulomb_coeff = T.coulomb_coeff;
            o.dt = T.dt;
            o.dt_over_tloss_pref = T.dt_over_tloss_pref;
            o.dtT_e = T.dtT_e;
            o.alpha = T.alpha;
            o.dpp_inv = on.inv;
            o.flags = kPreActive | (g.windowed ? kPreWindowed : 0) | (T.interp ? kPreInterp : 0) |
                      (on.fill ? kPreFill : 0);
            o.sl = g.sl;
            o.el = g.el;
            o.steps = g.steps;
        }
        P.pre[i] = o;
    }
}

// Dpp eta-cap scale of every tracer of the chunk with a segment in slot g0,
// from the spectra at the start of the segment (prepare_momentumdiff_cell_major,
// src/fp_shared_core.c:1032-1081, runs before either species evolves), one
// warp per tracer.  The energy sum is split over the lanes and combined by a
// shuffle tree, so it agrees with the reference's sequential sum to rounding.
__global__ void __launch_bounds__(128) eta_scale_kernel(FusedParams P, double *eta)
{
    const int lane = threadIdx.x & 31;
    const int tl = blockIdx.x * 4 + (threadIdx.x >> 5);
    const SnapArgs &a = P.a;
    if (tl >= P.nt) return;
    const int t = P.t0 + tl;
    const SegInfo g = segment_of(P, t, P.g0);
    if (!g.active) return;
    const Bg bg = load_bg(a, t, g);
    const double tacc_direct = segment_tacc(P.mp, a, g);
    const double mass = a.mass ? a.mass[t] : 0.0;
    const double *crp = a.crp + (size_t)t * NB, *cre = a.cre + (size_t)t * NB;
    double ecr = 0.0;
    for (int j = 2 + lane; j < NB - 2; j += 32) {
        const double ekp = P.gt.s[0].E[j] - kMp, vp = crp[j];
        if (ekp > 0.0 && isfinite(vp)) ecr += ekp * kGeV * vp * P.gt.s[0].dp[j];
        const double eke = P.gt.s[1].E[j] - kMe, ve = cre[j];
        if (eke > 0.0 && isfinite(ve)) ecr += eke * kGeV * ve * P.gt.s[1].dp[j];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) ecr += __shfl_xor_sync(kFull, ecr, off);
    if (lane == 0) eta[t] = eta_cap_scale_from_ecr(P.mp, bg, mass, tacc_direct, ecr);
}

// Secondary source of every segment of the chunk, cell-major:
// inje[m][je] = Gyr n_gas(t, segment) sum_{jp} N_p[m][jp] fqe[jp][je] + qepri[t][je]
// over the rows m = gi * nt + tl of np_seg -- a [rows x nb] . [nb x nb] FP64
// GEMM on the FP64 tensor cores (mma.sync m8n8k4 .f64: one instruction is
// 256 multiply-adds).  A 128 x 64 output tile per 256-thread block, each warp
// a 32 x 32 tile of 4 x 4 MMA fragments; k-tiles of 16 double-buffered in
// shared memory by cp.async.  The proton index starts at the first k-tile
// holding a nonzero weight for the block's columns; fqe is zero below
// np_min_qe[je] (prepare_secondary_kernel_flat, src/fp_shared_core.c:1453-1506),
// so the rounded-down start adds exact zeros only.
constexpr int kGM = 128, kGN = 64, kGK = 16;
// Row pitches chosen so that the fragment reads of a half warp (rows gid or
// tig, 4 x 4 lanes) land on 16 distinct bank pairs: 20 and 68 doubles.
constexpr int kGPitchA = kGK + 4;    // sA[m][k], 20 doubles per row
constexpr int kGPitchB = kGN + 4;    // sB[k][n], 68 doubles per row

struct GemmSmem {
    double A[2][kGM][kGPitchA];
    double B[2][kGK][kGPitchB];
};

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256, 2) secondary_kernel(FusedParams P)
{
    extern __shared__ double4 smem_raw[];
    GemmSmem &sm = *reinterpret_cast<GemmSmem *>(smem_raw);
    const SnapArgs &a = P.a;
    const int nrows = (P.g1 - P.g0) * P.nt;   // < 2^31, checked on the host
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;   // warp tile origin in the block tile
    const int gid = lane >> 2, tig = lane & 3;                // MMA fragment coordinates
    // column tile fastest, so the NB / kGN blocks of one row tile run together
    // and read their A tile from L2
    const int n0 = (int)(blockIdx.x % (NB / kGN)) * kGN;
    const int m0 = (int)(blockIdx.x / (NB / kGN)) * kGM;
    int jstart = NB;
    for (int i = 0; i < kGN; i++) jstart = min(jstart, P.np_min_qe[n0 + i]);
    jstart = max(jstart, P.gt.fqe_jp0);
    const int kbeg = (jstart / kGK) * kGK;

    // loader roles: A rows (4 chunks of 16 B per thread), B rows (2 chunks)
    auto load_tile = [&](int buf, int k0) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int q = tid + 256 * c;          // 0..1023: row q / 8, chunk q % 8
            const int r = q >> 3, ch = q & 7;
            const int m = m0 + r;
            const bool ok = m < nrows;
            const double *src = P.np_seg + (size_t)(ok ? m : 0) * NB + k0 + ch * 2;
            cp_async16(&sm.A[buf][r][ch * 2], src, ok);
        }
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int q = tid + 256 * c;          // 0..511: row q / 32, chunk q % 32
            const int r = q >> 5, ch = q & 31;
            const double *src = P.gt.fqe + (size_t)(k0 + r) * NB + n0 + ch * 2;
            cp_async16(&sm.B[buf][r][ch * 2], src, true);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

    if (kbeg < NB) load_tile(0, kbeg);
    int buf = 0;
#pragma unroll 1
    for (int k0 = kbeg; k0 < NB; k0 += kGK) {
        const bool more = k0 + kGK < NB;
        if (more) {
            load_tile(buf ^ 1, k0 + kGK);
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kGK; kk += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; i++) af[i] = sm.A[buf][wm + 8 * i + gid][kk + tig];
#pragma unroll
            for (int j = 0; j < 4; j++) bf[j] = sm.B[buf][kk + tig][wn + 8 * j + gid];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
        __syncthreads();
        buf ^= 1;
    }

    // epilogue: fragment (i, j) holds C[wm + 8i + gid][wn + 8j + 2 tig + {0, 1}]
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int m = m0 + wm + 8 * i + gid;
        if (m >= nrows) continue;
        const int gi = m / P.nt, tl = m - gi * P.nt;
        const int t = P.t0 + tl;
        const SegPre *__restrict__ pre = P.pre + (size_t)gi * P.nt + tl;
        if (!(pre->flags & kPreActive)) continue;
        const double ng = pre->n_gas;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int je = n0 + wn + 8 * j + 2 * tig;
            double q0 = 0.0, q1 = 0.0;
            if (a.qepri) {
                q0 = a.qepri[(size_t)t * NB + je];
                q1 = a.qepri[(size_t)t * NB + je + 1];
            }
            *reinterpret_cast<double2 *>(P.inje + (size_t)m * NB + je) =
                make_double2(acc[i][j][0] * kGyr * ng + q0, acc[i][j][1] * kGyr * ng + q1);
        }
    }
}

cudaError_t launch_secondary(Context &ctx, const FusedParams &P)
{
    constexpr size_t smem = sizeof(GemmSmem);
    // set once per process; thread-safe (function-local static initialisation)
    static const cudaError_t attr =
        cudaFuncSetAttribute(secondary_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (attr != cudaSuccess) return attr;
    const long long rows = (long long)(P.g1 - P.g0) * P.nt;
    if (rows > 0x7fffffffLL) return cudaErrorInvalidValue;
    const long long blocks = (rows + kGM - 1) / kGM * (NB / kGN);
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    secondary_kernel<<<(unsigned)blocks, 256, smem, ctx.stream>>>(P);
    return cudaGetLastError();
}

template <int S, bool ROWS>
cudaError_t launch_factor(Context &ctx, const FusedParams &P)
{
    constexpr size_t smem = (size_t)kTab * kTabStride * sizeof(double) + kFacWarps * sizeof(WarpSmem);
    // blocks per SM, per instantiation: found once (thread-safe static initialisation)
    struct Occupancy { cudaError_t e; int resident; };
    static const Occupancy occ = [] {
        Occupancy o{cudaSuccess, 0};
        o.e = cudaFuncSetAttribute(factor_kernel<S, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem);
        if (o.e == cudaSuccess)
            o.e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.resident, factor_kernel<S, ROWS>,
                                                                kFacWarps * 32, smem);
        return o;
    }();
    if (occ.e != cudaSuccess) return occ.e;
    if (occ.resident < 1) return cudaErrorInvalidConfiguration;
    const int resident = occ.resident;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    long long blocks = ((long long)P.nt + kFacWarps - 1) / kFacWarps;
    const long long full = (long long)nsm * resident;
    if (blocks > full) blocks = full;
    if (blocks < 1) return cudaSuccess;
    const cudaError_t ez = cudaMemsetAsync(P.work + S, 0, sizeof(unsigned), ctx.stream);
    if (ez != cudaSuccess) return ez;
    factor_kernel<S, ROWS><<<(unsigned)blocks, kFacWarps * 32, smem, ctx.stream>>>(P);
    return cudaGetLastError();
}

// One steps-kernel variant: solver and warps per block (1, 2 or 4), on the
// first `tracers` tracers of the chunk (all when <= 0).
template <int S, bool SRC, int SOLVER, int WPB>
cudaError_t launch_steps_variant(cudaStream_t st, const FusedParams &P, int tracers)
{
    const int n = tracers > 0 ? min(tracers, P.nt) : P.nt;
    const int blocks = (n + WPB - 1) / WPB;
    const size_t smem = SOLVER == kSolvePcr ? WPB * sizeof(PcrSmem)
                      : SOLVER == kSolveScanShared ? (size_t)WPB * kCoefSmemDoubles * sizeof(double)
                      : SOLVER == kSolveScanRhs    ? (size_t)WPB * kRhsSmemDoubles * sizeof(double)
                                                   : 0;
    if (smem > 48 * 1024) {
        static const cudaError_t attr = cudaFuncSetAttribute(steps_kernel<S, SRC, SOLVER, WPB>,
                                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (attr != cudaSuccess) return attr;
    }
    steps_kernel<S, SRC, SOLVER, WPB><<<blocks, WPB * 32, smem, st>>>(P);
    return cudaGetLastError();
}

// Variants the autotuner chooses between: (solver, warps per block).
constexpr int kStepVariants = CROMA_B200_STEPS_VARIANTS;
constexpr int kVariantSolver[kStepVariants] = {kSolveScan, kSolveScan, kSolveScanShared, kSolveScanShared,
                                               kSolvePcr, kSolveScanRhs, kSolveScanRhs, kSolveScan4,
                                               kSolveScan4};
constexpr int kVariantWpb[kStepVariants] = {1, 2, 1, 2, 1, 1, 2, 1, 2};

// Arithmetic families: variants of one family compute bit-identical results
// (the same operations in the same order; only where the constants live and
// how many warps share a block differ), so the tuner's timing-based choice
// within a family never changes a result.  0: the scan; 1: the short-chain
// scan; 2: PCR.
constexpr int kVariantFamily[kStepVariants] = {0, 0, 0, 0, 2, 0, 0, 1, 1};

// The family the tuner times: PCR when CROMA_CUDA_TRIDIAG=pcr, else the
// short-chain scan at 512 bins and more (measured faster there: its shorter
// shuffle chain outweighs its extra instructions at 8 warps per SM) and the
// scan below (where the short-chain form spills at the larger warp count).
int tune_family(int env) { return env == 2 ? 2 : (NB >= 512 ? 1 : 0); }

template <int S, bool SRC>
cudaError_t launch_variant(cudaStream_t st, const FusedParams &P, int v, int tracers)
{
    switch (v) {
    case 1: return launch_steps_variant<S, SRC, kSolveScan, 2>(st, P, tracers);
    case 2: return launch_steps_variant<S, SRC, kSolveScanShared, 1>(st, P, tracers);
    case 3: return launch_steps_variant<S, SRC, kSolveScanShared, 2>(st, P, tracers);
    case 4: return launch_steps_variant<S, SRC, kSolvePcr, 1>(st, P, tracers);
    case 5: return launch_steps_variant<S, SRC, kSolveScanRhs, 1>(st, P, tracers);
    case 6: return launch_steps_variant<S, SRC, kSolveScanRhs, 2>(st, P, tracers);
    case 7: return launch_steps_variant<S, SRC, kSolveScan4, 1>(st, P, tracers);
    case 8: return launch_steps_variant<S, SRC, kSolveScan4, 2>(st, P, tracers);
    default: return launch_steps_variant<S, SRC, kSolveScan, 1>(st, P, tracers);
    }
}

// CROMA_CUDA_TRIDIAG (src/fp_cuda_solver.cu:41-63 of the reference): "thomas"
// keeps the scan solvers, "pcr" forces PCR, unset lets the tuner choose.
int tridiag_env()
{
    const char *e = getenv("CROMA_CUDA_TRIDIAG");
    if (!e) e = getenv("FP_GPU_CUDA_TRIDIAG");
    if (!e) return 0;
    if (strcmp(e, "thomas") == 0) return 1;
    if (strcmp(e, "pcr") == 0) return 2;
    return 0;
}

// The autotuner: on the first chunk a context evolves, each admissible
// variant of the family tune_family names runs the chunk's first tracers (at
// most kTuneTracers) for their first 16 sub-steps on a copy of their spectra,
// timed with CUDA events; the fastest is kept for the context's species.  Results are recorded in
// ctx.tune.  kTuneTracers is several full waves of every variant (8 to 24
// warps per SM on 148 SMs): a sample below one wave favours the variants
// with more warps per SM, which lose at full size.  A calibration on the full
// sample is kept for the process (per species, source and
// CROMA_CUDA_TRIDIAG setting) and reused by later contexts with at least as
// many tracers; smaller chunks calibrate on themselves.
// CROMA_B200_STEPS_VARIANT = 0..8 fixes the variant (scan x1, scan x2, shared
// scan x1, shared scan x2, PCR, rhs-shared scan x1, rhs-shared scan x2,
// short-chain scan x1, short-chain scan x2)
// without calibrating, for reproducible profiles; unset or out of range: tune.
constexpr int kTuneTracers = 16384;
TuneState g_tune[2][2][3];   // [species][source][CROMA_CUDA_TRIDIAG: unset, thomas, pcr]
std::mutex g_tune_mu;

int fixed_variant_env()
{
    const char *e = getenv("CROMA_B200_STEPS_VARIANT");
    if (!e || !*e) return -1;
    const int v = atoi(e);
    return (v >= 0 && v < kStepVariants) ? v : -1;
}

template <int S>
int tune_steps(Context &ctx, const FusedParams &P, bool src)
{
    TuneState &tu = ctx.tune[S];
    const int fixed = fixed_variant_env();
    if (fixed >= 0) {
        tu.variant = fixed;
        tu.tuned = 1;
        return 0;
    }
    const int env = tridiag_env();
    const int T = min(P.nt, kTuneTracers), steps = 16;
    TuneState *shared = nullptr;
    if (T == kTuneTracers) {
        shared = &g_tune[S][src ? 1 : 0][env];
        std::lock_guard<std::mutex> lk(g_tune_mu);
        if (shared->tuned) {
            tu = *shared;
            return 0;
        }
    }
    double *scratch = nullptr;
    CROMA_CUDA(dev_alloc(ctx, &scratch, (size_t)T * NB * sizeof(double)));
    struct Free {
        Context &c;
        double *p;
        ~Free() { dev_free(c, p); }
    } guard{ctx, scratch};
    const double *real = (S == 0 ? P.a.crp : P.a.cre) + (size_t)P.t0 * NB;
    FusedParams Q = P;
    Q.cal_spec = scratch;
    Q.cal_steps = steps;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CROMA_CUDA(cudaEventCreate(&e0));
    CROMA_CUDA(cudaEventCreate(&e1));
    int best = -1;
    const int family = tune_family(env);
    for (int v = 0; v < kStepVariants; v++) {
        tu.ms[v] = -1.0;
        if (kVariantFamily[v] != family) continue;
        double ms_best = 1e30;
        for (int rep = 0; rep < 2; rep++) {   // the first run warms the code and L2
            CROMA_CUDA(cudaMemcpyAsync(scratch, real, (size_t)T * NB * sizeof(double), cudaMemcpyDeviceToDevice,
                                       ctx.stream));
            CROMA_CUDA(cudaEventRecord(e0, ctx.stream));
            CROMA_CUDA((src ? launch_variant<S, true>(ctx.stream, Q, v, T) : launch_variant<S, false>(ctx.stream, Q, v, T)));
            CROMA_CUDA(cudaEventRecord(e1, ctx.stream));
            CROMA_CUDA(cudaEventSynchronize(e1));
            float ms = 0.0f;
            CROMA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (rep == 1) ms_best = ms;
        }
        tu.ms[v] = ms_best;
        if (best < 0 || ms_best < tu.ms[best]) best = v;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    tu.variant = best < 0 ? 0 : best;
    tu.tuned = 1;
    tu.tracers = T;
    tu.steps = steps;
    if (shared) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        if (!shared->tuned) *shared = tu;
    }
    return 0;
}

template <int S>
cudaError_t launch_steps(Context &ctx, const FusedParams &P, bool src, bool perstep)
{
    const int blocks = (P.nt + kWarps - 1) / kWarps;
    if (perstep) {
        if (src) plain_steps_kernel<S, true><<<blocks, kWarps * 32, 0, ctx.stream>>>(P);
        else plain_steps_kernel<S, false><<<blocks, kWarps * 32, 0, ctx.stream>>>(P);
        return cudaGetLastError();
    }
    if (ctx.cfg.path == CROMA_PATH_FUSED_FP32R) {
        if (src) return launch_steps_variant<S, true, kSolveRefined, 1>(ctx.stream, P, 0);
        return launch_steps_variant<S, false, kSolveRefined, 1>(ctx.stream, P, 0);
    }
    if (!ctx.tune[S].tuned) {
        const int rc = tune_steps<S>(ctx, P, src);
        if (rc) return cudaErrorUnknown;
    }
    const int v = ctx.tune[S].variant;
    return src ? launch_variant<S, true>(ctx.stream, P, v, 0) : launch_variant<S, false>(ctx.stream, P, v, 0);
}

// Workspace budget of the fused path (factored matrices, segment-start
// proton spectra, segment sources); CROMA_B200_WORKSPACE_GB overrides it.
double workspace_budget_bytes()
{
    const char *s = getenv("CROMA_B200_WORKSPACE_GB");
    double gb = s ? atof(s) : 0.0;
    if (!(gb > 0.0)) gb = 24.0;
    return gb * 1e9;
}

}  // namespace

namespace {

struct WorkspaceShape {
    int nseg, sets;
    long long chunk;
    double per_tracer;
};

// The per-step path holds one segment slot at a time; the on-chip path all
// of a snapshot's slots.
WorkspaceShape workspace_shape(const ModelParams &mp, int cap, double workspace_cap, bool perstep)
{
    WorkspaceShape w;
    w.nseg = perstep ? 1
                     : (mp.interp_max_segments < 1 ? 1 : (mp.interp_max_segments > 64 ? 64 : mp.interp_max_segments));
    w.sets = mp.window_centred ? 2 : 1;
    w.per_tracer = 8.0 * NB * ((double)2 * w.nseg * w.sets * 3 + 2.0 * w.nseg) + (double)w.nseg * sizeof(SegPre);
    const double budget = workspace_cap > 0.0 ? workspace_cap : workspace_budget_bytes();
    w.chunk = (long long)(budget / w.per_tracer);
    if (w.chunk < 1) w.chunk = 1;
    if (w.chunk > cap) w.chunk = cap;
    return w;
}

}  // namespace

double fused_workspace_bytes(const ModelParams &mp, int cap, double workspace_cap, int path)
{
    const WorkspaceShape w = workspace_shape(mp, cap, workspace_cap, path == CROMA_PATH_PLAIN);
    return (double)w.chunk * w.per_tracer + 8.0 * cap;
}

int fused_reserve(Context &ctx, int cap)
{
    const WorkspaceShape w = workspace_shape(ctx.mp, cap, ctx.workspace_bytes, ctx.cfg.path == CROMA_PATH_PLAIN);
    const int nseg = w.nseg, sets = w.sets;
    const long long chunk = w.chunk;
    dev_free(ctx, ctx.d_inje);
    dev_free(ctx, ctx.d_eta_scale);
    dev_free(ctx, ctx.d_fac);
    dev_free(ctx, ctx.d_np_seg);
    dev_free(ctx, ctx.d_segpre);
    dev_free(ctx, ctx.d_work);
    ctx.d_inje = ctx.d_eta_scale = ctx.d_fac = ctx.d_np_seg = nullptr;
    ctx.d_segpre = nullptr;
    ctx.d_work = nullptr;
    ctx.fused_chunk = ctx.fused_nseg = ctx.fused_sets = 0;
    const size_t rows = (size_t)nseg * chunk * NB;
    CROMA_CUDA(dev_alloc(ctx, &ctx.d_fac, (size_t)2 * sets * rows * 3 * sizeof(double)));
    CROMA_CUDA(dev_alloc(ctx, &ctx.d_np_seg, rows * sizeof(double)));
    CROMA_CUDA(dev_alloc(ctx, &ctx.d_inje, rows * sizeof(double)));
    CROMA_CUDA(dev_alloc(ctx, &ctx.d_eta_scale, (size_t)cap * sizeof(double)));
    CROMA_CUDA(dev_alloc(ctx, &ctx.d_segpre, (size_t)nseg * chunk * sizeof(SegPre)));
    CROMA_CUDA(dev_alloc(ctx, &ctx.d_work, 2 * sizeof(unsigned)));
    ctx.fused_chunk = (int)chunk;
    ctx.fused_nseg = nseg;
    ctx.fused_sets = sets;
    return 0;
}

// Segments [g0, g1) of one tracer chunk: the eta-cap scales (if the cap is
// on), the factored matrices of both species, the proton steps, the
// secondary source, the electron steps.  perstep (the plain path, one slot):
// the raw rows of both species, the secondary source from the protons at the
// slot start, then the per-step kernels.
// Host-pipeline copies of one chunk's rows of one species: after an event on
// the compute stream, on the d2h stream.
static int pipe_download(Context &ctx, const FusedParams &P, cudaEvent_t ev, double *host, const double *dev)
{
    CROMA_CUDA(cudaEventRecord(ev, ctx.stream));
    CROMA_CUDA(cudaStreamWaitEvent(ctx.d2h_stream, ev, 0));
    const size_t off = (size_t)P.t0 * NB, bytes = (size_t)P.nt * NB * sizeof(double);
    CROMA_CUDA(cudaMemcpyAsync(host + off, dev + off, bytes, cudaMemcpyDeviceToHost, ctx.d2h_stream));
    return 0;
}

// pk >= 0 (host pipeline, all segments in one launch): the chunk's upload is
// awaited only before the first steps kernel -- the per-segment scalars and
// the factored rows do not read the spectra -- and the proton rows go back as
// soon as the proton steps are done.
static int fused_range(Context &ctx, FusedParams &P, int g0, int g1, bool perstep, int pk = -1)
{
    const SnapArgs &a = P.a;
    const int protons = ctx.mp.species_mask & CROMA_SPECIES_PROTON;
    const int electrons = ctx.mp.species_mask & CROMA_SPECIES_ELECTRON;
    const bool secondaries = protons && electrons;
    const bool cap = ctx.mp.eta_dpp_cap > 0.0 && isfinite(ctx.mp.eta_dpp_cap) && ctx.mp.dpp_model != kDppOff;
    if ((cap || perstep) && g1 != g0 + 1) {
        set_error("internal: the eta cap and the per-step path need one segment per launch");
        return -1;
    }
    P.g0 = g0;
    P.g1 = g1;
    P.eta_scale = nullptr;
    // protons at the segment start: recorded by the steps kernel, or (per
    // step, one slot) the chunk's resident rows themselves
    P.np_seg = !secondaries ? nullptr : (perstep ? a.crp + (size_t)P.t0 * NB : ctx.d_np_seg);
    P.inje = secondaries ? ctx.d_inje : nullptr;
    cudaEvent_t ev = nullptr;
    timed_begin(ctx, kKindCoeff, &ev);
    if (cap) {
        eta_scale_kernel<<<(P.nt + 3) / 4, 128, 0, ctx.stream>>>(P, ctx.d_eta_scale);
        ctx.last_launches += 1;
        P.eta_scale = ctx.d_eta_scale;
    }
    if (protons || electrons) {
        const long long total = (long long)(g1 - g0) * P.nt;
        int dev = 0, nsm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        long long blocks = (total + 255) / 256;
        if (blocks > 8LL * nsm) blocks = 8LL * nsm;
        seg_pre_kernel<<<(unsigned)blocks, 256, 0, ctx.stream>>>(P);
        ctx.last_launches += 1;
    }
    if (protons) {
        CROMA_CUDA((perstep ? launch_factor<0, true>(ctx, P) : launch_factor<0, false>(ctx, P)));
        ctx.last_launches += 1;
    }
    if (electrons) {
        CROMA_CUDA((perstep ? launch_factor<1, true>(ctx, P) : launch_factor<1, false>(ctx, P)));
        ctx.last_launches += 1;
    }
    timed_end(ctx, kKindCoeff, ev);
    if (pk >= 0) CROMA_CUDA(cudaStreamWaitEvent(ctx.stream, ctx.pipe_up[pk], 0));
    if (secondaries && perstep) {
        timed_begin(ctx, kKindSecondary, &ev);
        CROMA_CUDA(launch_secondary(ctx, P));
        timed_end(ctx, kKindSecondary, ev);
        ctx.last_launches += 1;
    }
    if (protons) {
        timed_begin(ctx, kKindEvolve, &ev);
        CROMA_CUDA(launch_steps<0>(ctx, P, a.qpi != nullptr, perstep));
        timed_end(ctx, kKindEvolve, ev);
        ctx.last_launches += 1;
    }
    if (pk >= 0 && ctx.pipe->down_p) {
        const int rc = pipe_download(ctx, P, ctx.pipe_done_p[pk], ctx.pipe->crp, a.crp);
        if (rc) return rc;
    }
    if (secondaries && !perstep) {
        timed_begin(ctx, kKindSecondary, &ev);
        CROMA_CUDA(launch_secondary(ctx, P));
        timed_end(ctx, kKindSecondary, ev);
        ctx.last_launches += 1;
    }
    if (electrons) {
        timed_begin(ctx, kKindEvolve, &ev);
        CROMA_CUDA(launch_steps<1>(ctx, P, secondaries || a.qepri != nullptr, perstep));
        timed_end(ctx, kKindEvolve, ev);
        ctx.last_launches += 1;
    }
    CROMA_CUDA(cudaGetLastError());
    return 0;
}

// Every segment slot of every tracer chunk.
static int fused_chunks(Context &ctx, FusedParams &P, int nslots, bool perstep)
{
    if (ctx.fused_chunk <= 0 || !ctx.d_fac) {
        set_error("fused workspace not reserved");
        return -1;
    }
    if ((perstep ? 1 : nslots) > ctx.fused_nseg) {
        set_error("internal: more segment slots than the fused workspace holds");
        return -1;
    }
    const bool windows = P.explicit_seg ? P.ex.windowed != 0 : ctx.mp.window_centred != 0;
    if (windows && ctx.fused_sets < 2) {
        set_error("internal: windowed segments without an off-coefficient workspace");
        return -1;
    }
    // the evolve kernels access rows with 32-byte vector loads and stores
    auto misaligned = [](const void *p) { return ((uintptr_t)p & 31u) != 0; };
    if (misaligned(P.a.crp) || misaligned(P.a.cre) || misaligned(P.a.qpi) || misaligned(P.a.qepri) ||
        misaligned(ctx.d_fac) || misaligned(ctx.d_inje) || misaligned(ctx.d_np_seg)) {
        set_error("internal: spectra, sources or workspace not 32-byte aligned");
        return -1;
    }
    const bool cap = ctx.mp.eta_dpp_cap > 0.0 && isfinite(ctx.mp.eta_dpp_cap) && ctx.mp.dpp_model != kDppOff;
    P.sets = ctx.fused_sets;
    P.fac = ctx.d_fac;
    P.pre = static_cast<SegPre *>(ctx.d_segpre);
    P.work = ctx.d_work;
    // chunks: the workspace's uniform split, or the host pipeline's bounds
    // (each within the workspace chunk), whose uploads gate the chunk and
    // whose downloads follow it
    const HostPipe *pipe = ctx.pipe;
    const int nchunk = pipe ? (int)pipe->bounds.size() - 1
                            : (P.a.ntracer + ctx.fused_chunk - 1) / ctx.fused_chunk;
    for (int k = 0; k < nchunk; k++) {
        P.t0 = pipe ? pipe->bounds[k] : k * ctx.fused_chunk;
        const int t1 = pipe ? pipe->bounds[k + 1]
                            : (P.a.ntracer - P.t0 < ctx.fused_chunk ? P.a.ntracer : P.t0 + ctx.fused_chunk);
        P.nt = t1 - P.t0;
        if (P.nt <= 0 || P.nt > ctx.fused_chunk) {
            set_error("internal: tracer chunk outside the fused workspace");
            return -1;
        }
        if (!cap && !perstep) {
            // one launch per kernel for the chunk: the upload wait and the
            // proton download sit inside, next to the kernels they gate
            const int rc = fused_range(ctx, P, 0, nslots, false, pipe ? k : -1);
            if (rc) return rc;
        } else {
            if (pipe) CROMA_CUDA(cudaStreamWaitEvent(ctx.stream, ctx.pipe_up[k], 0));
            for (int g = 0; g < nslots; g++) {
                const int rc = fused_range(ctx, P, g, g + 1, perstep);
                if (rc) return rc;
            }
            if (pipe && pipe->down_p) {
                const int rc = pipe_download(ctx, P, ctx.pipe_done_p[k], pipe->crp, P.a.crp);
                if (rc) return rc;
            }
        }
        if (pipe && pipe->down_e) {
            const int rc = pipe_download(ctx, P, ctx.pipe_done[k], pipe->cre, P.a.cre);
            if (rc) return rc;
        }
    }
    return 0;
}

int run_fused(Context &ctx, const SnapArgs &a)
{
    FusedParams P{};
    P.a = a;
    P.gt = ctx.gt;
    P.mp = ctx.mp;
    P.np_min_qe = ctx.d_np_min_qe;
    P.explicit_seg = 0;
    P.ex = SegInfo{};
    P.ic_stride = 0;
    const int nslots = ctx.mp.interp_max_segments < 1 ? 1
                     : (ctx.mp.interp_max_segments > 64 ? 64 : ctx.mp.interp_max_segments);
    return fused_chunks(ctx, P, nslots, ctx.cfg.path == CROMA_PATH_PLAIN);
}

int tuning_info(const Context &ctx, int species, int *solver, int *wpb)
{
    if (species < 0 || species > 1) return -1;
    const TuneState &t = ctx.tune[species];
    if (solver) *solver = kVariantSolver[t.variant];
    if (wpb) *wpb = kVariantWpb[t.variant];
    return t.tuned;
}

int run_fused_segment(Context &ctx, const SnapArgs &a, const SegInfo &ex, int ic_stride)
{
    FusedParams P{};
    P.a = a;
    P.gt = ctx.gt;
    P.mp = ctx.mp;
    P.np_min_qe = ctx.d_np_min_qe;
    P.explicit_seg = 1;
    P.ex = ex;
    P.ic_stride = ic_stride;
    return fused_chunks(ctx, P, 1, false);
}

}  // namespace croma
