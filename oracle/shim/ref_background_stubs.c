/*
 * Link-time stand-ins for the background loaders that src/tracer_fp_restart.c
 * calls from tracer_fp_restart_bg (src/tracer_fp_restart.c:30-134) -- the
 * HDF5 and synthetic background translation units are not part of the
 * checker build.  The checker only calls the checkpoint writer and reader of
 * that file, never tracer_fp_restart_bg; each stand-in reports failure.
 * Test infrastructure: nothing in the product links this file.
 */
#include <stdio.h>

#include "tracer_fp_background.h"
#include "tracer_fp_debug.h"

void tracer_copy_background_slot(int ntracer, const TracerFpBackgroundSlot *dst,
                                 const TracerFpBackgroundSlot *src)
{
    (void)ntracer; (void)dst; (void)src;
    fprintf(stderr, "oracle/_ref: tracer_copy_background_slot is not compiled into this checker\n");
}

int tracer_load_hdf5_raw_snapshot_slice(const TracerFpHdf5Meta *meta, int snap_id, long int tracer_start,
                                        const int *selected_offsets, int ntracer,
                                        TracerFpRawBackgroundSlot *raw)
{
    (void)meta; (void)snap_id; (void)tracer_start; (void)selected_offsets; (void)ntracer; (void)raw;
    return -1;
}

int tracer_prepare_background_from_raw(int ntracer, const TracerFpRawBackgroundSlot *prev_raw,
                                       const TracerFpRawBackgroundSlot *curr_raw,
                                       const TracerFpRawBackgroundSlot *next_raw, double z_prev,
                                       double z_curr, double z_next, int apply_temp_floor,
                                       int allow_curl_interp, TracerFpBackgroundSlot *out)
{
    (void)ntracer; (void)prev_raw; (void)curr_raw; (void)next_raw; (void)z_prev; (void)z_curr;
    (void)z_next; (void)apply_temp_floor; (void)allow_curl_interp; (void)out;
    return -1;
}

int tracer_fp_fill_background_snapshot_synthetic(int isnap, const double *z_snap, int ntracer,
                                                 const long int *tracer_ids, int ntracer_global, int nsnap,
                                                 TracerFpBackgroundSlot *slot)
{
    (void)isnap; (void)z_snap; (void)ntracer; (void)tracer_ids; (void)ntracer_global; (void)nsnap;
    (void)slot;
    return -1;
}
