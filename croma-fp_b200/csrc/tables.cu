// tables.cu -- one-time grid tables and the per-redshift inverse-Compton
// cooling rows.
//
// Host side (glibc, once per context): the momentum grids
// (momentum_bin, src/FP_Coef.c:291-330), the grid caches of
// src/FP_Coef.c:77-156 (p^2, exp(-1/p), Kamae sigma_pp, sigmoid, j_pp) and
// the grid-only factors the kernels reuse.  These are the same host-side
// tables the reference's CUDA workspace uploads (fp_cuda_workspace.cu:253-433).
//
// Device side: the secondary-electron weights (prepare_secondary_kernel_flat,
// src/fp_shared_core.c:1453-1506) and the IC cooling row integrals
// (rad_IC_cool / b_IC, src/FP_Coef.c:361-375, 480-539).  The CMB photon
// energy bounds (a scalar Newton iteration per redshift, FP_Coef.c:414-436)
// and the outer abscissae are evaluated on the host and shared by all bins.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "croma_ctx.cuh"
#include "croma_hadronic.cuh"

namespace croma {

namespace {

// ---------------------------------------------------------------------
// Secondary-electron weights
// ---------------------------------------------------------------------
__global__ void qe_values_kernel(const double *Ee, const double *pp, const double *beta_p,
                                 double *vals)   // [je][jp]
{
    const int jp = blockIdx.x * blockDim.x + threadIdx.x;
    const int je = blockIdx.y;
    if (jp >= NB) return;
    double v = qe_kernel(Ee[je], pp[jp]) * beta_p[jp];
    if (isnan(v)) v = 0.0;
    vals[(size_t)je * NB + jp] = v;
}

__global__ void qe_weights_kernel(const double *vals, const double *dp_p, double *fqe,
                                  int *np_min_qe)
{
    const int je = blockIdx.x * blockDim.x + threadIdx.x;
    if (je >= NB) return;
    const double *v = vals + (size_t)je * NB;
    int jmin = 1;
    for (int jp = 1; jp < NB; jp++)
        if (v[jp] < 1.0e-80) jmin = jp;
    int jp0 = jmin;
    if (jp0 < 1) jp0 = 1;
    if (jp0 > NB) jp0 = NB;
    for (int jp = 0; jp < NB; jp++) {
        double w = 0.0;
        if (jp0 < NB) {
            if (jp == jp0 - 1) w = 0.5 * v[jp] * dp_p[jp0];
            else if (jp >= jp0 && jp < NB - 1) w = 0.5 * v[jp] * (dp_p[jp] + dp_p[jp + 1]);
            else if (jp == NB - 1 && jp >= jp0) w = 0.5 * v[jp] * dp_p[jp];
        }
        fqe[(size_t)jp * NB + je] = w;
    }
    np_min_qe[je] = (jp0 < NB) ? (jp0 - 1) : NB;
}

// ---------------------------------------------------------------------
// IC cooling: one block per electron momentum (nb bins, then pm1, pp1).
// outer[i] are the CMB photon energies e0_i (i = 0..nout), shared.
// ---------------------------------------------------------------------
constexpr int kIcMaxOuter = 2048;

__global__ void __launch_bounds__(512) ic_row_kernel(IcConsts icc, const double *p_e, double pm1, double pp1,
                              const double *outer, int nout, double z, double *row)
{
    __shared__ double s_n[kIcMaxOuter + 1];
    __shared__ double s_ic2[kIcMaxOuter + 1];
    const int j = blockIdx.x;
    const double p = (j < NB) ? p_e[j] : (j == NB ? pm1 : pp1);
    const double gamma = sqrt(1.0 + p * p);
    for (int i = threadIdx.x; i <= nout; i += blockDim.x) {
        const double e0 = outer[i];
        const double emax = gamma * 4.0 * e0 * gamma / (1.0 + 4.0 * e0 * gamma);
        s_ic2[i] = b_ic_integrand(e0, gamma, e0, emax);
        s_n[i] = cmb_density(icc, e0, z);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double integral = 0.0;
        for (int i = 0; i < nout; i++) {
            const double deps0 = outer[i + 1] - outer[i];
            integral = integral + 0.5 * (s_n[i] * s_ic2[i] + s_n[i + 1] * s_ic2[i + 1]) * deps0;
        }
        row[j] = integral * kGyr;
    }
}

// cmb_photon_energy_bounds, FP_Coef.c:414-436, on the host.
int cmb_bounds(const IcConsts &k, double z, double *emin, double *emax)
{
    const double delta = pow(10.0, -5.5);
    const double meg = 9.11 * pow(10.0, -28.0), cl = 3.0e+10, T0 = 2.725;
    const double kb = 1.38 * pow(10.0, -16.0);
    const double epsp = kb / (meg * cl * cl) * T0 * (1.0 + z);
    const double peak = cmb_density(k, epsp, z);
    double out[2];
    const double start[2] = {0.01 * epsp, 10.0 * epsp};
    for (int s = 0; s < 2; s++) {
        double epsnew = start[s], eps = 1.0;
        int it = 0;
        while (fabs(epsnew - eps) > delta * eps) {
            if (++it > 100000) return -1;
            eps = epsnew;
            epsnew = eps - (cmb_density(k, eps, z) - peak * delta) / cmb_density_deps(k, eps, z);
        }
        out[s] = epsnew;
    }
    *emin = out[0];
    *emax = out[1];
    return 0;
}

}  // namespace

int build_tables(Context &ctx)
{
    const CromaB200Config &c = ctx.cfg;
    const int n = NB;
    std::vector<double> beta_p(n);
    if (ctx.grid_given) {
        for (int j = 0; j < n; j++) beta_p[j] = ctx.h_p[0][j] / sqrt(1.0 + ctx.h_p[0][j] * ctx.h_p[0][j]);
    } else {
        // ---- momentum grids: momentum_bin, FP_Coef.c:291-330 ----
        for (int s = 0; s < 2; s++) {
            ctx.h_p[s].assign(n, 0.0);
            ctx.h_dp[s].assign(n, 0.0);
            ctx.h_E[s].assign(n, 0.0);
        }
        double da = (c.pmax - c.pmin) / (double)n, a = c.pmin - da;
        ctx.h_pm1[0] = pow(10.0, a);
        for (int j = 0; j < n; j++) {
            a = a + da;
            const double p = pow(10.0, a);
            ctx.h_p[0][j] = p;
            ctx.h_E[0][j] = kMp * sqrt(1.0 + p * p);
            beta_p[j] = p / sqrt(1.0 + p * p);
        }
        a = a + da;
        ctx.h_pp1[0] = pow(10.0, a);
        for (int j = 1; j < n - 1; j++) ctx.h_dp[0][j] = 0.5 * (ctx.h_p[0][j + 1] - ctx.h_p[0][j - 1]);
        ctx.h_dp[0][0] = 0.5 * (ctx.h_p[0][1] - ctx.h_pm1[0]);
        ctx.h_dp[0][n - 1] = 0.5 * (pow(10.0, a + da) - ctx.h_p[0][n - 2]);

        da = (c.pemax - c.pemin) / (double)n;
        a = c.pemin - da;
        ctx.h_pm1[1] = pow(10.0, a);
        for (int j = 0; j < n; j++) {
            a += da;
            const double p = pow(10.0, a);
            ctx.h_p[1][j] = p;
            ctx.h_E[1][j] = kMe * sqrt(1.0 + p * p);
        }
        a += da;
        ctx.h_pp1[1] = pow(10.0, a);
        for (int j = 1; j < n - 1; j++) ctx.h_dp[1][j] = 0.5 * (ctx.h_p[1][j + 1] - ctx.h_p[1][j - 1]);
        ctx.h_dp[1][0] = 0.5 * (ctx.h_p[1][1] - ctx.h_pm1[1]);
        ctx.h_dp[1][n - 1] = 0.5 * (pow(10.0, a + da) - ctx.h_p[1][n - 2]);
    }

    // ---- caches, FP_Coef.c:77-156 and the grid-only kinematics ----
    enum { T_P, T_DP, T_E, T_P2, T_CUT, T_2P, T_EXPE, T_IDX, T_IDXL, T_IDXR, T_DXF, T_RFF, T_PER };   // per species
    const int nspecies_arrays = T_PER * 2;
    // cp_Ep, cp_kin, cp_inv_betap2, sig_eff, ce_beta2, cp_inv2mpkin, ce_inv_beta2, ce_logp
    const int n_extra = 8;
    const size_t tab_doubles = (size_t)(nspecies_arrays + n_extra) * n + (size_t)n * n;
    std::vector<double> h(tab_doubles, 0.0);
    auto arr = [&](int k) { return h.data() + (size_t)k * n; };
    for (int s = 0; s < 2; s++) {
        double *P = arr(s * T_PER + T_P), *DP = arr(s * T_PER + T_DP), *E = arr(s * T_PER + T_E);
        double *P2 = arr(s * T_PER + T_P2), *CUT = arr(s * T_PER + T_CUT);
        double *TWO = arr(s * T_PER + T_2P), *EXPE = arr(s * T_PER + T_EXPE);
        double *IDX = arr(s * T_PER + T_IDX), *IDXL = arr(s * T_PER + T_IDXL), *IDXR = arr(s * T_PER + T_IDXR);
        double *DXF = arr(s * T_PER + T_DXF), *RFF = arr(s * T_PER + T_RFF);
        for (int j = 0; j < n; j++) {
            P[j] = ctx.h_p[s][j];
            DP[j] = ctx.h_dp[s][j];
            E[j] = ctx.h_E[s][j];
            P2[j] = P[j] * P[j];
            CUT[j] = exp(-1.0 / P[j]);
            TWO[j] = 2.0 / P[j];
            EXPE[j] = (s == 0) ? exp(-E[j] / kEpMax) : 1.0;
            IDX[j] = 1.0 / DP[j];
        }
        for (int j = 0; j < n; j++) {
            IDXL[j] = (j >= 1) ? 1.0 / (ctx.h_p[s][j] - ctx.h_p[s][j - 1]) : 0.0;
            IDXR[j] = (j <= n - 2) ? 1.0 / (ctx.h_p[s][j + 1] - ctx.h_p[s][j]) : 0.0;
            DXF[j] = (j <= n - 2) ? ctx.h_p[s][j + 1] - ctx.h_p[s][j] : 0.0;
        }
        // face j of the filled Dpp form: Dpp_j = kappa * p_j^2 expE_j exp(-1/p_j)
        // with kappa = dpp_inv * scale shared by the segment, so the face's
        // dx / (Dpp_j + Dpp_j+1) is this grid factor over kappa
        for (int j = 0; j < n; j++) {
            const double gl = P2[j] * EXPE[j] * CUT[j];
            const double gr = (j <= n - 2) ? P2[j + 1] * EXPE[j + 1] * CUT[j + 1] : 0.0;
            RFF[j] = (j <= n - 2) ? DXF[j] / (gl + gr) : 0.0;
        }
    }
    double *cpEp = arr(nspecies_arrays + 0), *cpKin = arr(nspecies_arrays + 1);
    double *cpIb = arr(nspecies_arrays + 2), *sigEff = arr(nspecies_arrays + 3);
    double *ceB2 = arr(nspecies_arrays + 4), *cpI2 = arr(nspecies_arrays + 5);
    double *ceIB2 = arr(nspecies_arrays + 6);
    double *ceLogp = arr(nspecies_arrays + 7);
    std::vector<double> sigma(n), sigmoid(n);
    for (int j = 0; j < n; j++) sigma[j] = pp_pion_xsec(2, kMp * ctx.h_p[0][j]);
    int j_pp = 0;
    for (int j = 0; j < n - 100; j++)
        if (j_pp == 0 && sigma[j] > 0.0) j_pp = j;
    j_pp += 2;
    if (j_pp < 0) j_pp = 0;
    if (j_pp >= n) j_pp = n - 1;
    const double p_pp = ctx.h_p[0][j_pp];
    for (int j = 0; j < n; j++) sigmoid[j] = 1.0 / (1.0 + exp(-5.0 * (ctx.h_p[0][j] - p_pp)));
    for (int j = 0; j < n; j++) {
        const double p = ctx.h_p[0][j], p2 = p * p;
        const double gamma = sqrt(1.0 + p2);
        cpEp[j] = gamma * kMp - kMp;
        cpKin[j] = gamma - 1.0;
        cpIb[j] = 1.0 / (p2 / (1.0 + p2));
        double sg = (j > j_pp) ? sigma[j] : sigma[j_pp];
        sg *= sigmoid[j];
        sigEff[j] = sg;
        cpI2[j] = 1.0 / (2.0 * kMp * cpKin[j]);
        const double pe2 = ctx.h_p[1][j] * ctx.h_p[1][j];
        ceB2[j] = pe2 / (1.0 + pe2);
        ceIB2[j] = 1.0 / ceB2[j];
        ceLogp[j] = log(ctx.h_p[1][j]);
    }

    // ---- device allocation ----
    dev_free(ctx, ctx.d_tables);
    dev_free(ctx, ctx.d_np_min_qe);
    ctx.d_tables = nullptr;
    ctx.d_np_min_qe = nullptr;
    CROMA_CUDA(dev_alloc(ctx, &ctx.d_tables, tab_doubles * sizeof(double)));
    double *d = ctx.d_tables;
    auto darr = [&](int k) { return d + (size_t)k * n; };
    for (int s = 0; s < 2; s++) {
        SpeciesTables &st = ctx.gt.s[s];
        st.p = darr(s * T_PER + T_P);
        st.dp = darr(s * T_PER + T_DP);
        st.E = darr(s * T_PER + T_E);
        st.p2 = darr(s * T_PER + T_P2);
        st.exp_cut = darr(s * T_PER + T_CUT);
        st.two_over_p = darr(s * T_PER + T_2P);
        st.expE = darr(s * T_PER + T_EXPE);
        st.inv_dx = darr(s * T_PER + T_IDX);
        st.inv_dxl = darr(s * T_PER + T_IDXL);
        st.inv_dxr = darr(s * T_PER + T_IDXR);
        st.dxf = darr(s * T_PER + T_DXF);
        st.face_rf = darr(s * T_PER + T_RFF);
        st.pm1 = ctx.h_pm1[s];
        st.pp1 = ctx.h_pp1[s];
        st.pm1_p2 = st.pm1 * st.pm1;
        st.pp1_p2 = st.pp1 * st.pp1;
        st.pm1_exp_cut = exp(-1.0 / st.pm1);
        st.pp1_exp_cut = exp(-1.0 / st.pp1);
        st.expE_m1 = exp(-kMp * sqrt(1.0 + st.pm1 * st.pm1) / kEpMax);
        st.expE_p1 = exp(-kMp * sqrt(1.0 + st.pp1 * st.pp1) / kEpMax);
    }
    ctx.gt.cp_Ep = darr(nspecies_arrays + 0);
    ctx.gt.cp_kin = darr(nspecies_arrays + 1);
    ctx.gt.cp_inv_betap2 = darr(nspecies_arrays + 2);
    ctx.gt.sig_eff = darr(nspecies_arrays + 3);
    ctx.gt.ce_beta2 = darr(nspecies_arrays + 4);
    ctx.gt.cp_inv2mpkin = darr(nspecies_arrays + 5);
    ctx.gt.ce_inv_beta2 = darr(nspecies_arrays + 6);
    ctx.gt.ce_logp = darr(nspecies_arrays + 7);
    for (int k = 0; k < 2; k++) {
        const double p = k == 0 ? ctx.h_pm1[0] : ctx.h_pp1[0], p2 = p * p;
        const double gamma = sqrt(1.0 + p2);
        const double Ep = gamma * kMp - kMp, kin = gamma - 1.0, ib = 1.0 / (p2 / (1.0 + p2));
        if (k == 0) { ctx.gt.cpm1_Ep = Ep; ctx.gt.cpm1_kin = kin; ctx.gt.cpm1_inv_betap2 = ib; }
        else { ctx.gt.cpp1_Ep = Ep; ctx.gt.cpp1_kin = kin; ctx.gt.cpp1_inv_betap2 = ib; }
    }
    {
        const double m2 = ctx.h_pm1[1] * ctx.h_pm1[1], p2 = ctx.h_pp1[1] * ctx.h_pp1[1];
        ctx.gt.cem1_beta2 = m2 / (1.0 + m2);
        ctx.gt.cep1_beta2 = p2 / (1.0 + p2);
    }
    ctx.gt.fqe = d + (size_t)(nspecies_arrays + n_extra) * n;
    ctx.gt.nb = n;
    CROMA_CUDA(cudaMemcpyAsync(d, h.data(), (size_t)(nspecies_arrays + n_extra) * n * sizeof(double),
                               cudaMemcpyHostToDevice, ctx.stream));

    // ---- IC constants (FP_Coef.c:402, 410-412) ----
    {
        const double meg = 9.11e-28;
        ctx.icc.cmb_pref = 8.0 * kPi * kC * kC * kC * pow(meg / kHPlanck, 3.0);
        ctx.icc.cmb_pref_d = 8.0 * kPi * kC * kC * kC * pow(meg / 6.63e-27, 3.0);
        ctx.icc.k_d = 1.38 * pow(10.0, -16.0);
        ctx.icc.log10_90 = 90.0 * log(10.0);
    }

    // ---- secondary-electron weights on the device ----
    {
        double *d_vals = nullptr, *d_aux = nullptr;
        int *d_npmin = nullptr;
        CROMA_CUDA(dev_alloc(ctx, &d_vals, (size_t)n * n * sizeof(double)));
        CROMA_CUDA(dev_alloc(ctx, &d_aux, (size_t)n * 2 * sizeof(double)));
        CROMA_CUDA(dev_alloc(ctx, &d_npmin, (size_t)n * sizeof(int)));
        CROMA_CUDA(cudaMemcpyAsync(d_aux, beta_p.data(), n * sizeof(double), cudaMemcpyHostToDevice,
                                   ctx.stream));
        dim3 g((n + 127) / 128, n);
        qe_values_kernel<<<g, 128, 0, ctx.stream>>>(ctx.gt.s[1].E, ctx.gt.s[0].p, d_aux, d_vals);
        qe_weights_kernel<<<(n + 127) / 128, 128, 0, ctx.stream>>>(d_vals, ctx.gt.s[0].dp,
                                                                   (double *)ctx.gt.fqe, d_npmin);
        CROMA_CUDA(cudaGetLastError());
        ctx.h_fqe.assign((size_t)n * n, 0.0);
        ctx.h_np_min_qe.assign(n, 0);
        CROMA_CUDA(cudaMemcpyAsync(ctx.h_fqe.data(), ctx.gt.fqe, (size_t)n * n * sizeof(double),
                                   cudaMemcpyDeviceToHost, ctx.stream));
        CROMA_CUDA(cudaMemcpyAsync(ctx.h_np_min_qe.data(), d_npmin, n * sizeof(int),
                                   cudaMemcpyDeviceToHost, ctx.stream));
        CROMA_CUDA(cudaStreamSynchronize(ctx.stream));
        dev_free(ctx, d_vals);
        dev_free(ctx, d_aux);
        ctx.d_np_min_qe = d_npmin;
        // first proton bin any electron bin draws from (fp_shared_core.c:1615-1623)
        int jp0 = n;
        for (int je = 0; je < n; je++) {
            int j0 = ctx.h_np_min_qe[je];
            if (j0 < 0) j0 = 0;
            if (j0 < jp0) jp0 = j0;
        }
        ctx.gt.fqe_jp0 = jp0;
    }
    return 0;
}

int ic_rows(Context &ctx, double z, double *d_out)
{
    double emin = 0.0, emax = 0.0;
    if (cmb_bounds(ctx.icc, z, &emin, &emax) != 0) {
        set_error("CMB photon-energy bound iteration did not converge");
        return -2;
    }
    // outer abscissae of b_IC (FP_Coef.c:480-511), accumulated as there
    const double da = 0.50e-1;
    const int N = (int)round((log10(emax) - log10(emin)) / da);
    if (N < 0 || N > kIcMaxOuter) {
        set_error("IC outer grid out of range");
        return -2;
    }
    if (!ctx.h_ic_stage) {
        ctx.h_ic_stage = acquire_ic_stage();
        if (!ctx.h_ic_stage) {
            set_error("page-locked IC staging allocation failed");
            return -4;
        }
        for (int k = 0; k < 2; k++)
            CROMA_CUDA(cudaEventCreateWithFlags(&ctx.ic_stage_ev[k], cudaEventDisableTiming));
    }
    const int k = ctx.ic_stage_next;
    ctx.ic_stage_next ^= 1;
    CROMA_CUDA(cudaEventSynchronize(ctx.ic_stage_ev[k]));   // the copy that last read this slot
    double *outer = ctx.h_ic_stage + (size_t)k * (kIcMaxOuter + 1);
    double a = log10(emin);
    outer[0] = emin;
    for (int i = 1; i <= N; i++) {
        a = a + da;
        outer[i] = pow(10.0, a);
    }
    double *d_outer = d_out + NB + 2;   // scratch tail reserved after the row
    CROMA_CUDA(cudaMemcpyAsync(d_outer, outer, (N + 1) * sizeof(double), cudaMemcpyHostToDevice,
                               ctx.stream));
    CROMA_CUDA(cudaEventRecord(ctx.ic_stage_ev[k], ctx.stream));
    ic_row_kernel<<<NB + 2, 512, 0, ctx.stream>>>(ctx.icc, ctx.gt.s[1].p, ctx.h_pm1[1], ctx.h_pp1[1],
                                                  d_outer, N, z, d_out);
    CROMA_CUDA(cudaGetLastError());
    return 0;
}

void free_ic_stage(Context &ctx)
{
    for (int k = 0; k < 2; k++) {
        if (ctx.ic_stage_ev[k]) cudaEventDestroy(ctx.ic_stage_ev[k]);
        ctx.ic_stage_ev[k] = nullptr;
    }
    if (ctx.h_ic_stage) release_ic_stage(ctx.h_ic_stage);
    ctx.h_ic_stage = nullptr;
}

namespace {
std::mutex g_stage_mu;
std::vector<double *> g_stage_free;   // released staging rows, kept for the process
}  // namespace

double *acquire_ic_stage()
{
    {
        std::lock_guard<std::mutex> lk(g_stage_mu);
        if (!g_stage_free.empty()) {
            double *p = g_stage_free.back();
            g_stage_free.pop_back();
            return p;
        }
    }
    double *p = nullptr;
    if (cudaMallocHost(&p, 2 * (size_t)(kIcMaxOuter + 1) * sizeof(double)) != cudaSuccess) return nullptr;
    return p;
}

void release_ic_stage(double *p)
{
    std::lock_guard<std::mutex> lk(g_stage_mu);
    g_stage_free.push_back(p);
}

}  // namespace croma
