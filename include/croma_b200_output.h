/*
 * croma_b200_output.h -- output files and checkpoints of the B200 tracer
 * Fokker-Planck library in the reference's on-disk formats
 * (src/tracer_fp_output.c, src/tracer_fp_restart.c of kosukenishiwaki/croma-fp),
 * written from host arrays or straight from a context's device-resident
 * spectra.
 *
 * Files of one rank:
 *   tile mode    <dir>/<stem>_tile_coreNN.bin   [nslab][nrow][ncol] doubles
 *                (tracer_fp_tile_open / _write_cr / _write_emit, :362-519)
 *   mapped mode  <dir>/<stem>_coreNN.bin        [nrow][nslab * ncol] doubles
 *                (tracer_fp_map_open, tracer_fp_write_cr_map / _emit_map,
 *                :251-332, :607-663)
 * with the reference's stems and slab counts: CRE / CRP over nsnap + 1 slabs
 * of nb columns (slab 0 = the initial state), eSyn / eIC / eGamma / eNu over
 * nsnap slabs.  A file is created at its full size (ftruncate +
 * posix_fallocate) or, with resume_existing, reopened after its size is
 * checked.  Rows are tracers.  With output_per_cc each row is scaled by
 * rho_gcc / (mass_msun * 1.99e33) (0 where either is not positive), the
 * reference's output_volume_factor (:177-189).
 *
 * Checkpoint: <dir>/checkpoint_rankNN.bin, the 72-byte TracerFpCheckpointHeader
 * (magic "TFPCHK1", version 1; include/tracer_fp_types.h:356-371), the
 * tracer ids, then the proton and electron spectra cell-major; written to
 * "<path>.tmp", fsync'ed and renamed (tracer_fp_ckpt_write, :143-203).  Reading
 * checks every header field and the tracer order (tracer_fp_ckpt_read,
 * :205-262).
 *
 * Return codes as in croma_b200.h (0 ok, -1 invalid argument or state,
 * -3 CUDA error, -5 I/O error); croma_b200_last_error() describes failures
 * of the calling thread.
 */
#ifndef CROMA_B200_OUTPUT_H
#define CROMA_B200_OUTPUT_H

#include <stddef.h>

#include "croma_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CromaB200Output CromaB200Output;

enum { CROMA_OUTPUT_TILE = 0, CROMA_OUTPUT_MAPPED = 1 };

/* Create (or, with resume_existing, reopen) one output file. */
int croma_b200_output_open(const char *dir, const char *stem, int mpi_rank, int mode, size_t nslab,
                           size_t nrow, size_t ncol, int resume_existing, CromaB200Output **out);

/* Slab `slab` from host rows [nrow][ncol] (cell-major).  rho_gcc / mass_msun
 * [nrow] are read only with output_per_cc.  Synchronous. */
int croma_b200_output_write(CromaB200Output *out, size_t slab, const double *rows, const double *rho_gcc,
                            const double *mass_msun, int output_per_cc);

/* Slab `slab` of the electron (and, if crp_out is not NULL, proton) spectra
 * resident in ctx, at the point the context stream has reached: the rows
 * (scaled by the volume factor with output_per_cc, from the host array
 * rho_gcc [ntracer] and the context's tracer masses) are staged in device
 * memory on the context stream, copied to page-locked host memory on a copy
 * stream and written by the file's writer thread, so the next snapshots run
 * while the data travels.  Returns once the work is queued; the host array
 * rho_gcc may be reused on return.  croma_b200_output_flush waits for it. */
int croma_b200_output_write_state(CromaB200Context *ctx, CromaB200Output *cre_out, CromaB200Output *crp_out,
                                  size_t slab, const double *rho_gcc, int output_per_cc);

/* Wait for the queued writes of this file; returns the first error. */
int croma_b200_output_flush(CromaB200Output *out);
/* Flush, fsync and close; out is freed. */
int croma_b200_output_close(CromaB200Output *out);

typedef struct {
    const char *dir;
    int mpi_rank;
    int world_size;
    int ntracer;
    int ntracer_global;
    int nsnap;
    int nfreq;
    int nsnp_i;              /* the reference's snapshot index range (params.c nsnp_i / nsnp_f) */
    int nsnp_f;
    int completed_snapshot;  /* written; ignored when reading */
    long tracer_start;
    const int *tracer_ids;   /* [ntracer] */
} CromaB200Checkpoint;

/* Checkpoint of host spectra crp [ntracer][np], cre [ntracer][npe]. */
int croma_b200_checkpoint_write_host(const CromaB200Checkpoint *ck, int np_bins, int npe_bins,
                                     const double *crp, const double *cre);
/* Checkpoint of the spectra resident in ctx (ntracer must equal its tracer count). */
int croma_b200_checkpoint_write(CromaB200Context *ctx, const CromaB200Checkpoint *ck);
/* Read into host arrays; *completed_snapshot receives the header's value. */
int croma_b200_checkpoint_read_host(const CromaB200Checkpoint *ck, int np_bins, int npe_bins, double *crp,
                                    double *cre, int *completed_snapshot);
/* Read into ctx as set_state(crp, cre) would (sources and flags zero, the
 * masses kept). */
int croma_b200_checkpoint_read(CromaB200Context *ctx, const CromaB200Checkpoint *ck, int *completed_snapshot);

#ifdef __cplusplus
}
#endif

#endif
