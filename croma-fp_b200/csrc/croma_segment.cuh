// croma_segment.cuh -- per-tracer segment set-up shared by the evolve
// kernels: which sub-steps a coefficient segment covers, the interpolated
// background, the Dpp model choice, the eta cap and the per-bin loss and
// diffusion terms.  Internal header (device code).
//
//   segments   tracer_fp_batch_execute_bucket, src/tracer_fp_batch.c:651-827
//   Dpp        prepare_momentumdiff_cell_major, src/fp_shared_core.c:1241-1317,
//              momentumdiff_* src/FP_Coef.c:680-849
//   eta cap    fp_apply_eta_dpp_cap_cell, src/fp_shared_core.c:1032-1081
//   losses     prepare_{crp,cre}_losses_1d, src/fp_shared_core.c:729-842
#pragma once

#include "croma_ctx.cuh"

namespace croma {

struct SegInfo {
    int active;
    int nsub, nseg, b, e, steps;
    int windowed, sl, el;
    double alpha, dt;
};

// Segment `slot` of a tracer with the given schedule entries.
__device__ __forceinline__ SegInfo seg_info_of(int nseg, int nsub, int non, int slot, double dt_snap)
{
    SegInfo g{};
    g.nseg = nseg;
    if (slot >= g.nseg) return g;
    g.nsub = nsub;
    // slot < 64 and nsub <= 1e6 (the sub-step ceiling), so 32-bit products suffice
    g.b = (slot * g.nsub) / g.nseg;
    g.e = ((slot + 1) * g.nsub) / g.nseg;
    g.steps = g.e - g.b;
    if (g.steps <= 0) return g;
    g.active = 1;
    g.alpha = (g.nseg > 1) ? ((double)slot + 0.5) / (double)g.nseg : 0.0;
    const int on_start = (g.nsub - non) / 2, on_end = on_start + non;
    const int sob = on_start > g.b ? on_start : g.b;
    int soe = on_end < g.e ? on_end : g.e;
    if (soe < sob) soe = sob;
    g.windowed = ((soe - sob) < g.steps) ? 1 : 0;
    g.sl = sob - g.b;
    g.el = g.sl + (soe - sob);
    g.dt = dt_snap / (double)g.nsub;
    return g;
}

__device__ __forceinline__ SegInfo seg_info(const Schedule &s, int t, int slot, double dt_snap)
{
    const int nseg = s.nseg[t];
    if (slot >= nseg) {
        SegInfo g{};
        g.nseg = nseg;
        return g;
    }
    return seg_info_of(nseg, s.nsub[t], s.non[t], slot, dt_snap);
}


__device__ __forceinline__ double lerp(double c, double n, double a)
{
    if (a <= 0.0) return c;
    if (a >= 1.0) return n;
    return c + a * (n - c);
}

struct Bg {
    double n_gas, kbt, b_field, divv, lturb, dv, cs, beta;
};

__device__ __forceinline__ Bg load_bg(const SnapArgs &a, int t, const SegInfo &g)
{
    const size_t N = (size_t)a.ntracer;
    double v[kNbg];
#pragma unroll
    for (int f = 0; f < kNbg; f++) {
        const double c = a.bg_curr[f * N + t];
        v[f] = (g.nseg > 1) ? lerp(c, a.bg_next[f * N + t], g.alpha) : c;
    }
    return Bg{v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]};
}

// Background of segment g from the raw rows of the current and next snapshot.
__device__ __forceinline__ Bg lerp_bg(const double cur[kNbg], const double nxt[kNbg], const SegInfo &g)
{
    double v[kNbg];
#pragma unroll
    for (int f = 0; f < kNbg; f++) v[f] = (g.nseg > 1) ? lerp(cur[f], nxt[f], g.alpha) : cur[f];
    return Bg{v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]};
}

// Dpp scale for one cell: momentumdiff_* (FP_Coef.c:680-849) via the model
// choice of prepare_momentumdiff_cell_major (fp_shared_core.c:1241-1317).
// Returns inv = 1/(4 t_acc) with fill = 1, or fill = 0 for the "off" form
// p^2 / (4 * 1e5).
struct DppForm {
    int fill;
    double inv;
};

__device__ inline DppForm dpp_form(const ModelParams &mp, int model, const Bg &bg, double tacc_direct)
{
    DppForm f{0, 0.0};
    if (!(bg.dv > 0.0) || !isfinite(bg.dv) || model == kDppOff) return f;
    if (model == kDppAsa) {
        const double mach = effective_mach(mp.mach_limit, bg.dv, bg.cs);
        if (mach <= 0.0 || bg.beta <= 0.0) return f;
        f.fill = 1;
        f.inv = 1.0 / (4.0 * tacc_asa(mp.psi3, bg.lturb * kMpc, bg.cs, mach, bg.beta));
    } else if (model == kDppTtd) {
        const double mach = effective_mach(mp.mach_limit, bg.dv, bg.cs);
        if (mach <= 0.0 || bg.dv <= 0.0) return f;
        f.fill = 1;
        f.inv = 1.0 / (4.0 * tacc_ttd(mp.ttd_brunetti16, bg.lturb * kMpc, bg.cs, mach, bg.dv));
    } else if (model == kDppDirect) {
        if (!(tacc_direct > 0.0) || !isfinite(tacc_direct)) return f;
        f.fill = 1;
        f.inv = 1.0 / (4.0 * tacc_direct);
    }
    return f;
}

// fp_apply_eta_dpp_cap_cell (fp_shared_core.c:1032-1081): the factor by
// which the "on" Dpp is scaled (1 when the cap does not act).
// The cap from a given CR energy sum ecr (erg): the tail of the routine below.
__device__ inline double eta_cap_scale_from_ecr(const ModelParams &mp, const Bg &bg, double mass,
                                                double tacc_direct, double ecr)
{
    if (!(mp.eta_dpp_cap > 0.0) || !isfinite(mp.eta_dpp_cap)) return 1.0;
    if (!(mass > 0.0) || !(bg.lturb > 0.0) || !(bg.dv > 0.0)) return 1.0;
    double tacc = 0.0;
    if (bg.lturb > 0.0 && bg.cs > 0.0) {
        double mach = bg.dv / bg.cs;
        if (mach < 0.0) mach = 0.0;
        if (mp.mach_limit > 0.0 && mach > mp.mach_limit) mach = mp.mach_limit;
        if (mach > 0.0) {
            if (mp.dpp_model == kDppAsa) tacc = (bg.beta > 0.0) ? tacc_asa(mp.psi3, bg.lturb * kMpc, bg.cs, mach, bg.beta) : 0.0;
            else if (mp.dpp_model == kDppTtd) tacc = tacc_ttd(mp.ttd_brunetti16, bg.lturb * kMpc, bg.cs, mach, bg.dv);
            else if (mp.dpp_model == kDppDirect) tacc = (tacc_direct > 0.0 && isfinite(tacc_direct)) ? tacc_direct : 0.0;
        }
    }
    if (!(tacc > 0.0) || !isfinite(tacc)) return 1.0;
    const double qturb = 0.5 * mass * kMsun * bg.dv * bg.dv * bg.dv / (bg.lturb * kMpc);
    if (!(ecr > 0.0) || !(qturb > 0.0) || !isfinite(ecr) || !isfinite(qturb)) return 1.0;
    const double eta = ecr / (qturb * tacc * kGyr);
    if (!(eta > mp.eta_dpp_cap) || !isfinite(eta)) return 1.0;
    return mp.eta_dpp_cap / eta;
}

__device__ inline double eta_cap_scale(const ModelParams &mp, const GridTables &gt, const Bg &bg,
                                double mass, double tacc_direct, const double *crp,
                                const double *cre, size_t stride)
{
    if (!(mp.eta_dpp_cap > 0.0) || !isfinite(mp.eta_dpp_cap)) return 1.0;
    if (!(mass > 0.0) || !(bg.lturb > 0.0) || !(bg.dv > 0.0)) return 1.0;
    // fp_momentumdiff_tacc_gyr (fp_shared_core.c:993-1030)
    double tacc = 0.0;
    if (bg.lturb > 0.0 && bg.cs > 0.0) {
        double mach = bg.dv / bg.cs;
        if (mach < 0.0) mach = 0.0;
        if (mp.mach_limit > 0.0 && mach > mp.mach_limit) mach = mp.mach_limit;
        if (mach > 0.0) {
            if (mp.dpp_model == kDppAsa) tacc = (bg.beta > 0.0) ? tacc_asa(mp.psi3, bg.lturb * kMpc, bg.cs, mach, bg.beta) : 0.0;
            else if (mp.dpp_model == kDppTtd) tacc = tacc_ttd(mp.ttd_brunetti16, bg.lturb * kMpc, bg.cs, mach, bg.dv);
            else if (mp.dpp_model == kDppDirect) tacc = (tacc_direct > 0.0 && isfinite(tacc_direct)) ? tacc_direct : 0.0;
        }
    }
    if (!(tacc > 0.0) || !isfinite(tacc)) return 1.0;
    double ecr = 0.0;
    for (int j = 2; j < NB - 2; j++) {
        const double ek = gt.s[0].E[j] - kMp, v = crp[j * stride];
        if (ek > 0.0 && isfinite(v)) ecr += ek * kGeV * v * gt.s[0].dp[j];
    }
    for (int j = 2; j < NB - 2; j++) {
        const double ek = gt.s[1].E[j] - kMe, v = cre[j * stride];
        if (ek > 0.0 && isfinite(v)) ecr += ek * kGeV * v * gt.s[1].dp[j];
    }
    const double qturb = 0.5 * mass * kMsun * bg.dv * bg.dv * bg.dv / (bg.lturb * kMpc);
    if (!(ecr > 0.0) || !(qturb > 0.0) || !isfinite(ecr) || !isfinite(qturb)) return 1.0;
    const double eta = ecr / (qturb * tacc * kGyr);
    if (!(eta > mp.eta_dpp_cap) || !isfinite(eta)) return 1.0;
    return mp.eta_dpp_cap / eta;
}

struct Terms {
    double B, C, dtT;
};

// One species of one tracer: loss and diffusion terms per bin.
struct SpeciesTerms {
    const GridTables *gt;
    int s;
    double n_gas, kbt, adiab;       // adiab = divv_loss / 3
    double synch_coeff, coulomb_coeff, tloss_pref;
    const double *ric;              // electron IC row (current), null for protons
    const double *ric_next;
    double alpha;
    int interp;
    DppForm dform;
    double dpp_scale;
    double dt;

    __device__ double radp(int j) const
    {
        const SpeciesTables &st = gt->s[s];
        const double p = st.p[j];
        if (s == 0)
            return coulomb_p(n_gas, kbt, gt->cp_Ep[j], gt->cp_kin[j], gt->cp_inv_betap2[j]) + adiab * p;
        const double pe2 = st.p2[j];
        const double r = interp ? lerp(ric[j], ric_next[j], alpha) : ric[j];
        const double coulomb = coulomb_coeff * (1.0 + log(p / n_gas) / 74.8) / gt->ce_beta2[j];
        return synch_coeff * pe2 + r + coulomb + adiab * p;
    }
    __device__ double dpp_at(int j) const
    {
        const SpeciesTables &st = gt->s[s];
        double d;
        if (!this->dform.fill) d = st.p2[j] * (1.0 / (4.0 * 1.0e+5));
        else if (s == 0) d = st.p2[j] * this->dform.inv * st.expE[j] * st.exp_cut[j];
        else d = st.p2[j] * this->dform.inv * st.exp_cut[j];
        return d * dpp_scale;
    }
    __device__ Terms at(int j) const
    {
        const double D = dpp_at(j);
        Terms t;
        t.B = radp(j) - gt->s[s].two_over_p[j] * D;
        t.C = D;
        t.dtT = (s == 0) ? dt / (tloss_pref / gt->sig_eff[j]) : dt / 1.0e+100;
        return t;
    }
};


// Per-tracer scalars of one species for one segment.
__device__ __forceinline__ SpeciesTerms make_species_terms(const GridTables &gt, int s, const Bg &bg,
                                                           int dis, const SnapArgs &a, const SegInfo &g)
{
    SpeciesTerms T;
    const double divv_loss = dis ? 0.0 : bg.divv;
    T.gt = &gt;
    T.s = s;
    T.n_gas = bg.n_gas;
    T.kbt = bg.kbt;
    T.adiab = 1.0 / 3.0 * divv_loss;
    const double b_ratio = bg.b_field * 1.0e+6 / 3.2;
    T.synch_coeff = 4.8e-4 * b_ratio * b_ratio * 9.11e-28 * 3.0e+10 * 3.1536e+16;
    T.coulomb_coeff = 3.05e-29 * bg.n_gas * kC * kGyr / (kMe * kGeV);
    T.tloss_pref = 1.0 / (0.5 * kC * bg.n_gas) / kGyr;
    T.ric = a.ic_curr;
    T.ric_next = a.ic_next;
    T.alpha = g.alpha;
    T.interp = g.nseg > 1;
    T.dt = g.dt;
    T.dform = DppForm{0, 0.0};
    T.dpp_scale = 1.0;
    return T;
}

// fused.cu: one caller-defined segment for every tracer (ic_stride 0: one
// shared IC row; otherwise per-tracer rows, momentum-major [nb][ic_stride]).
int run_fused_segment(Context &ctx, const SnapArgs &a, const SegInfo &ex, int ic_stride);

// cpu_direct_tacc_value (src/tracer_fp_batch.c:44-62): the direct t_acc of
// a segment, switched to t_acc_off before t_off.
__device__ __forceinline__ double segment_tacc(const ModelParams &mp, const SnapArgs &a, const SegInfo &g)
{
    double tacc = mp.t_acc_direct_gyr;
    if (mp.dpp_model == kDppDirect && isfinite(tacc) && tacc > 0.0 && isfinite(mp.t_off_gyr) &&
        mp.t_off_gyr > 0.0 && isfinite(mp.t_acc_off_gyr) && mp.t_acc_off_gyr > 0.0) {
        const double tmid = a.elapsed + ((double)g.b + 0.5 * (double)g.steps) * g.dt;
        if (tmid < mp.t_off_gyr) tacc = mp.t_acc_off_gyr;
    }
    return tacc;
}

}  // namespace croma
