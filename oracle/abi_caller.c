/*
 * A C caller of the drop-in ABI, compiled against the REFERENCE's own
 * headers (include/fp_cuda_backend.h, include/fp_shared_core.h,
 * include/params.h of kosukenishiwaki/croma-fp, -Dnp=-Dnpe=N) and linked to
 * this repository's libcroma_b200_np<N>.so -- the way CROMA's host binds the
 * library.  Test infrastructure: tests/test_gpu_ref_abi.py
 * writes the inputs of one (bucket, segment) call as CROMA's snapshot driver
 * makes it (include/tracer_fp_solve.inc:1341-1463), this program runs
 *   cuda_pipeline_workspace_create -> cuda_rank_state_upload ->
 *   run_tracer_pipeline (gather/scatter through the rank state) ->
 *   cuda_rank_state_download -> cuda_pipeline_workspace_destroy
 * and writes the downloaded spectra; the test compares them with the oracle.
 *
 *   abi_caller <input file> <output file>
 *
 * Input (native doubles unless stated): int32 ncell, nstep, windowed, on0,
 * on1, dpp_model, ttd_model; double dt, t_acc_direct, eta_cap; the proton
 * then electron grid (p[N], dp[N], E[N], pm1, pp1); bg[8][ncell]; ric[N][ncell];
 * m1[ncell]; p1[ncell]; mass[ncell]; uint8 dis[ncell]; crp, cre, qpi, qepri
 * [ncell][N] cell-major.  Output: crp then cre [ncell][N].
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fp_cuda_backend.h"

/* standalone model switches of this library (no counterpart in the reference) */
int croma_b200_set_model(int dpp_model, int ttd_tacc_model, double t_acc_direct_gyr, double eta_dpp_cap);
const char *croma_b200_last_error(void);

static int rd(FILE *f, void *p, size_t n)
{
    return fread(p, 1, n, f) == n ? 0 : -1;
}

static double *rdd(FILE *f, size_t n)
{
    double *p = (double *)malloc(n * sizeof(double));
    if (p && rd(f, p, n * sizeof(double))) { free(p); return 0; }
    return p;
}

static int rd_grid(FILE *f, CRspectrum *g)
{
    memset(g, 0, sizeof *g);
    if (rd(f, g->p, sizeof g->p) || rd(f, g->dp, sizeof g->dp) || rd(f, g->E, sizeof g->E)) return -1;
    if (rd(f, &g->pm1, sizeof(double)) || rd(f, &g->pp1, sizeof(double))) return -1;
    return 0;
}

int main(int argc, char **argv)
{
    int hdr[7];
    double dhdr[3];
    static CRspectrum gp, ge;
    FILE *f;
    if (argc != 3) { fprintf(stderr, "usage: abi_caller <in> <out>\n"); return 2; }
    f = fopen(argv[1], "rb");
    if (!f || rd(f, hdr, sizeof hdr) || rd(f, dhdr, sizeof dhdr) || rd_grid(f, &gp) || rd_grid(f, &ge)) {
        fprintf(stderr, "abi_caller: bad input\n");
        return 2;
    }
    const int ncell = hdr[0], nstep = hdr[1];
    double *bg = rdd(f, 8 * (size_t)ncell), *ric = rdd(f, (size_t)npe * ncell);
    double *m1 = rdd(f, ncell), *p1 = rdd(f, ncell), *mass = rdd(f, ncell);
    unsigned char *dis = (unsigned char *)malloc(ncell);
    if (!dis || rd(f, dis, ncell)) return 2;
    double *crp = rdd(f, (size_t)ncell * np), *cre = rdd(f, (size_t)ncell * npe);
    double *qpi = rdd(f, (size_t)ncell * np), *qepri = rdd(f, (size_t)ncell * npe);
    fclose(f);
    if (!bg || !ric || !m1 || !p1 || !mass || !crp || !cre || !qpi || !qepri) return 2;
    if (croma_b200_set_model(hdr[5], hdr[6], dhdr[1], dhdr[2]) != 0) return 3;

    FpCoeffBatchInput ci;
    memset(&ci, 0, sizeof ci);
    ci.ncell = ncell;
    ci.epmax = 1.0e7;
    ci.n_gas = bg; ci.kbt = bg + ncell; ci.b_field = bg + 2 * ncell; ci.divv_gyr = bg + 3 * ncell;
    ci.l_turb_mpc = bg + 4 * ncell; ci.dv_imc = bg + 5 * ncell; ci.cs = bg + 6 * ncell; ci.beta_pl = bg + 7 * ncell;
    ci.rad_ic_batch = ric; ci.rad_ic_m1 = m1; ci.rad_ic_p1 = p1;
    ci.tracer_mass_msun = mass;
    ci.disable_adiabatic = dis;

    FpCudaPipelineWorkspace *ws = cuda_pipeline_workspace_create();
    if (!ws) { fprintf(stderr, "abi_caller: %s\n", croma_b200_last_error()); return 3; }
    int rc = cuda_rank_state_upload(ws, ncell, qpi, qepri, crp, cre, 0);
    int *idx = (int *)malloc((size_t)ncell * sizeof(int));
    for (int i = 0; i < ncell; i++) idx[i] = i;
    FpCudaPipelineInput in;
    memset(&in, 0, sizeof in);
    in.ncell = ncell;
    in.nstep = nstep;
    in.fp_cadence_steps = in.diff_cadence_steps = in.adv_cadence_steps = 1;
    in.use_windowed_reacc = hdr[2];
    in.on_start_step = hdr[3];
    in.on_end_step = hdr[4];
    in.dt = dhdr[0];
    in.epmax = 1.0e7;
    in.psi_value = 0.5;
    in.mach_limit_value = 0.5;
    in.transport_mode = FP_CUDA_TRANSPORT_FUSED_SUBSTEPS;
    in.crp_grid = &gp;
    in.cre_grid = &ge;
    in.coeff_in = &ci;
    in.rank_state_indices = idx;
    in.gather_rank_state = 1;
    in.scatter_rank_state = 1;
    in.workspace = ws;
    FpCudaPipelineTimes times;
    memset(&times, 0, sizeof times);
    if (rc == 0) rc = run_tracer_pipeline(&in, 0, 0, 0, 0, 0, 0, &times);
    if (rc == 0) rc = cuda_rank_state_download(ws, ncell, crp, cre, 0);
    if (rc != 0) fprintf(stderr, "abi_caller: rc %d: %s\n", rc, croma_b200_last_error());
    cuda_pipeline_workspace_destroy(ws);
    if (rc != 0) return 4;
    f = fopen(argv[2], "wb");
    if (!f) return 2;
    fwrite(crp, sizeof(double), (size_t)ncell * np, f);
    fwrite(cre, sizeof(double), (size_t)ncell * npe, f);
    fclose(f);
    printf("abi_caller ok: %d cells, %d steps, solve %.3f ms\n", ncell, nstep, times.solve_ms);
    return 0;
}
