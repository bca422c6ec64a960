// output.cu -- output files and checkpoints in the reference's on-disk
// formats (include/croma_b200_output.h), from host arrays or from a
// context's device-resident spectra.
//
// Device path: the rows are staged in device memory by a kernel on the
// context stream (a copy, or the volume-factor scaling), copied to one of
// two page-locked host slots on the file's copy stream, and written by the
// file's writer thread with pwrite once the copy's event has fired.  The
// context stream waits only for the previous copy out of the device staging
// buffer before restaging it, so snapshots keep running while data travels
// over PCIe and to the file system.
#include <fcntl.h>
#include <sys/stat.h>
#include <sys/types.h>
#include <unistd.h>

#include <cerrno>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "croma_ctx.cuh"
#include "../../include/croma_b200_output.h"

struct CromaB200Context {
    croma::Context impl;
};

namespace croma {
namespace {

constexpr double kMsun = 1.99e+33;   // M_sun of the reference (src/CONSTANTS.c:6)

int io_fail(const std::string &what)
{
    set_error(what + ": " + strerror(errno));
    return -5;
}

// ensure_output_dir (src/tracer_fp_output.c:96-107)
int ensure_dir(const char *path)
{
    struct stat st;
    if (!path || !*path) return -1;
    if (stat(path, &st) == 0) return S_ISDIR(st.st_mode) ? 0 : -1;
    if (mkdir(path, 0755) == 0) return 0;
    if (stat(path, &st) == 0 && S_ISDIR(st.st_mode)) return 0;
    return -1;
}

int pwrite_all(int fd, const void *buf, size_t nbyte, off_t offset)
{
    const char *p = static_cast<const char *>(buf);
    size_t done = 0;
    while (done < nbyte) {
        const ssize_t n = pwrite(fd, p + done, nbyte - done, offset + (off_t)done);
        if (n < 0) {
            if (errno == EINTR) continue;
            return -1;
        }
        if (n == 0) {
            errno = EIO;
            return -1;
        }
        done += (size_t)n;
    }
    return 0;
}

// output_volume_factor (src/tracer_fp_output.c:177-189)
__host__ __device__ inline double volume_factor(const double *rho, const double *mass, size_t i, int per_cc)
{
    if (!per_cc) return 1.0;
    if (!rho || !mass) return 1.0;
    if (!(rho[i] > 0.0) || !(mass[i] > 0.0)) return 0.0;
    return rho[i] / (mass[i] * kMsun);
}

// dst[t][j] = src[t][j] * factor(t): the staging of one slab
__global__ void stage_rows_kernel(const double *src, double *dst, size_t nrow, int ncol, const double *rho,
                                  const double *mass, int per_cc)
{
    const size_t total = nrow * (size_t)ncol;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t t = i / (size_t)ncol;
        dst[i] = per_cc ? src[i] * volume_factor(rho, mass, t, per_cc) : src[i];
    }
}

struct Job {
    int slot;
    size_t slab;
    cudaEvent_t copied;
};

}  // namespace
}  // namespace croma

using namespace croma;

struct CromaB200Output {
    int fd = -1;
    int mode = CROMA_OUTPUT_TILE;
    size_t nslab = 0, nrow = 0, ncol = 0, nbyte = 0;
    std::string path;

    // device path, set up on the first write_state
    int device = -1;
    bool dev_ready = false;
    cudaStream_t copy_stream = nullptr;
    double *d_stage = nullptr, *d_rho = nullptr;
    double *h_slot[2] = {nullptr, nullptr};
    cudaEvent_t ev_staged = nullptr, ev_copied[2] = {nullptr, nullptr};
    bool slot_busy[2] = {false, false};
    int next_slot = 0;
    int last_slot = -1;

    std::mutex mu;
    std::condition_variable cv;
    std::deque<Job> queue;
    std::thread writer;
    bool stop = false;
    int err = 0;
    std::string err_msg;
    size_t pending = 0;   // jobs queued or being written
};

namespace croma {
namespace {

// One slab from host rows: the tile file's contiguous slab, or each row's
// column block of the mapped file.  The rows are already scaled.
int write_slab_rows(CromaB200Output *o, size_t slab, const double *rows)
{
    if (o->mode == CROMA_OUTPUT_TILE) {
        const size_t slab_values = o->nrow * o->ncol;
        if (pwrite_all(o->fd, rows, slab_values * sizeof(double), (off_t)(slab * slab_values * sizeof(double))) != 0)
            return io_fail("write " + o->path);
        return 0;
    }
    const size_t row_values = o->nslab * o->ncol;
    for (size_t r = 0; r < o->nrow; r++) {
        const size_t first = r * row_values + slab * o->ncol;
        if (pwrite_all(o->fd, rows + r * o->ncol, o->ncol * sizeof(double), (off_t)(first * sizeof(double))) != 0)
            return io_fail("write " + o->path);
    }
    return 0;
}

void writer_main(CromaB200Output *o)
{
    cudaSetDevice(o->device);
    for (;;) {
        Job j;
        {
            std::unique_lock<std::mutex> lk(o->mu);
            o->cv.wait(lk, [&] { return o->stop || !o->queue.empty(); });
            if (o->queue.empty()) return;
            j = o->queue.front();
            o->queue.pop_front();
        }
        int rc = 0;
        std::string msg;
        const cudaError_t e = cudaEventSynchronize(j.copied);
        if (e != cudaSuccess) {
            rc = -3;
            msg = std::string("CUDA error ") + cudaGetErrorName(e) + " in the output copy of " + o->path;
        } else {
            rc = write_slab_rows(o, j.slab, o->h_slot[j.slot]);
            if (rc) msg = "write " + o->path + ": " + strerror(errno);
        }
        {
            std::lock_guard<std::mutex> lk(o->mu);
            o->slot_busy[j.slot] = false;
            o->pending -= 1;
            if (rc && !o->err) {
                o->err = rc;
                o->err_msg = msg;
            }
        }
        o->cv.notify_all();
    }
}

int check_slab(const CromaB200Output *o, size_t slab)
{
    if (!o || o->fd < 0) { set_error("output not open"); return -1; }
    if (slab >= o->nslab) { set_error("slab index beyond the file's slabs"); return -1; }
    return 0;
}

// Device resources of one file for rows of ncol doubles, on ctx's device.
int ensure_device_path(CromaB200Output *o, Context &c)
{
    if (o->device >= 0) {
        if (o->device != c.device) { set_error("output file used with contexts on two devices"); return -1; }
        if (!o->dev_ready) { set_error("the output's device buffers could not be set up"); return -1; }
        return 0;
    }
    o->device = c.device;   // from here on close releases whatever was allocated
    const size_t bytes = o->nrow * o->ncol * sizeof(double);
    CROMA_CUDA(cudaStreamCreateWithFlags(&o->copy_stream, cudaStreamNonBlocking));
    CROMA_CUDA(cudaMalloc(&o->d_stage, bytes));
    CROMA_CUDA(cudaMalloc(&o->d_rho, o->nrow * sizeof(double)));
    for (int s = 0; s < 2; s++) {
        CROMA_CUDA(cudaMallocHost(&o->h_slot[s], bytes));
        CROMA_CUDA(cudaEventCreateWithFlags(&o->ev_copied[s], cudaEventDisableTiming));
    }
    CROMA_CUDA(cudaEventCreateWithFlags(&o->ev_staged, cudaEventDisableTiming));
    o->writer = std::thread(writer_main, o);
    o->dev_ready = true;
    return 0;
}

// Queue one slab of device rows src [nrow][ncol] of ctx for writing.
int queue_device_slab(CromaB200Output *o, Context &c, const double *src, size_t slab, const double *rho_host,
                      int per_cc)
{
    int rc = ensure_device_path(o, c);
    if (rc) return rc;
    // a free host slot (the writer releases it once written)
    int s;
    {
        std::unique_lock<std::mutex> lk(o->mu);
        s = o->next_slot;
        o->cv.wait(lk, [&] { return !o->slot_busy[s]; });
        if (o->err) { set_error(o->err_msg); return o->err; }
        o->slot_busy[s] = true;
        o->pending += 1;
        o->next_slot ^= 1;
    }
    // the device staging buffer is free once the previous copy out of it is done
    if (o->last_slot >= 0) CROMA_CUDA(cudaStreamWaitEvent(c.stream, o->ev_copied[o->last_slot], 0));
    const bool scale = per_cc && rho_host;
    if (scale)
        CROMA_CUDA(cudaMemcpyAsync(o->d_rho, rho_host, o->nrow * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    const size_t total = o->nrow * o->ncol;
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c.device);
    size_t blocks = (total + 255) / 256;
    if (blocks > (size_t)nsm * 8) blocks = (size_t)nsm * 8;
    if (blocks < 1) blocks = 1;
    stage_rows_kernel<<<(unsigned)blocks, 256, 0, c.stream>>>(src, o->d_stage, o->nrow, (int)o->ncol,
                                                              scale ? o->d_rho : nullptr, c.d_mass, scale ? 1 : 0);
    CROMA_CUDA(cudaGetLastError());
    c.last_launches += 1;
    CROMA_CUDA(cudaEventRecord(o->ev_staged, c.stream));
    CROMA_CUDA(cudaStreamWaitEvent(o->copy_stream, o->ev_staged, 0));
    CROMA_CUDA(cudaMemcpyAsync(o->h_slot[s], o->d_stage, total * sizeof(double), cudaMemcpyDeviceToHost,
                               o->copy_stream));
    CROMA_CUDA(cudaEventRecord(o->ev_copied[s], o->copy_stream));
    o->last_slot = s;
    {
        std::lock_guard<std::mutex> lk(o->mu);
        o->queue.push_back(Job{s, slab, o->ev_copied[s]});
    }
    o->cv.notify_all();
    return 0;
}

// TracerFpCheckpointHeader (include/tracer_fp_types.h:356-371)
struct CkptHeader {
    char magic[16];
    int version;
    int mpi_rank;
    int world_size;
    int ntracer;
    int ntracer_global;
    int nsnap;
    int nfreq;
    int np_bins;
    int npe_bins;
    int nsnp_i_value;
    int nsnp_f_value;
    int completed_snapshot;
    long int tracer_start;
};
static_assert(sizeof(CkptHeader) == 72, "checkpoint header layout");

std::string ckpt_path(const char *dir, int rank)
{
    char buf[4096];
    snprintf(buf, sizeof buf, "%s/checkpoint_rank%02d.bin", dir, rank);
    return buf;
}

int check_ckpt(const CromaB200Checkpoint *ck)
{
    if (!ck || !ck->dir || !*ck->dir || !ck->tracer_ids || ck->ntracer <= 0) {
        set_error("invalid checkpoint arguments");
        return -1;
    }
    return 0;
}

}  // namespace
}  // namespace croma

extern "C" {

int croma_b200_output_open(const char *dir, const char *stem, int mpi_rank, int mode, size_t nslab, size_t nrow,
                           size_t ncol, int resume_existing, CromaB200Output **out)
{
    if (!out || !dir || !*dir || !stem || (mode != CROMA_OUTPUT_TILE && mode != CROMA_OUTPUT_MAPPED) ||
        ncol == 0 || (mode == CROMA_OUTPUT_TILE && (nslab == 0 || nrow == 0)) ||
        (mode == CROMA_OUTPUT_MAPPED && nslab == 0)) {
        set_error("invalid output arguments");
        return -1;
    }
    *out = nullptr;
    if (nrow != 0 && (nslab > ((size_t)-1) / nrow || nslab * nrow > ((size_t)-1) / ncol / sizeof(double))) {
        set_error("output size overflows");
        return -1;
    }
    auto *o = new CromaB200Output();
    o->mode = mode;
    o->nslab = nslab;
    o->nrow = nrow;
    o->ncol = ncol;
    o->nbyte = nslab * nrow * ncol * sizeof(double);
    char buf[4096];
    if (mode == CROMA_OUTPUT_TILE) snprintf(buf, sizeof buf, "%s/%s_tile_core%02d.bin", dir, stem, mpi_rank);
    else snprintf(buf, sizeof buf, "%s/%s_core%02d.bin", dir, stem, mpi_rank);
    o->path = buf;
    o->fd = resume_existing ? open(o->path.c_str(), O_RDWR) : open(o->path.c_str(), O_RDWR | O_CREAT | O_TRUNC, 0644);
    int rc = 0;
    if (o->fd < 0) {
        rc = io_fail("open " + o->path);
    } else if (resume_existing) {
        struct stat st;
        if (fstat(o->fd, &st) != 0) {
            rc = io_fail("stat " + o->path);
        } else if ((size_t)st.st_size != o->nbyte) {
            set_error("existing output " + o->path + " has size " + std::to_string((long long)st.st_size) +
                      ", expected " + std::to_string(o->nbyte));
            rc = -1;
        }
    } else {
        if (ftruncate(o->fd, (off_t)o->nbyte) != 0) {
            rc = io_fail("truncate " + o->path);
        } else if (o->nbyte > 0) {
            const int e = posix_fallocate(o->fd, 0, (off_t)o->nbyte);
            if (e != 0) {
                errno = e;
                rc = io_fail("allocate " + o->path);
            }
        }
    }
    if (rc) {
        if (o->fd >= 0) close(o->fd);
        delete o;
        return rc;
    }
    *out = o;
    return 0;
}

int croma_b200_output_write(CromaB200Output *o, size_t slab, const double *rows, const double *rho_gcc,
                            const double *mass_msun, int output_per_cc)
{
    int rc = check_slab(o, slab);
    if (rc) return rc;
    if (!rows && o->nrow) { set_error("null rows"); return -1; }
    if (!output_per_cc) return write_slab_rows(o, slab, rows);
    std::vector<double> tmp(o->nrow * o->ncol);
    for (size_t t = 0; t < o->nrow; t++) {
        const double f = volume_factor(rho_gcc, mass_msun, t, output_per_cc);
        for (size_t j = 0; j < o->ncol; j++) tmp[t * o->ncol + j] = rows[t * o->ncol + j] * f;
    }
    return write_slab_rows(o, slab, tmp.data());
}

int croma_b200_output_write_state(CromaB200Context *h, CromaB200Output *cre_out, CromaB200Output *crp_out,
                                  size_t slab, const double *rho_gcc, int output_per_cc)
{
    if (!h || !cre_out) { set_error("invalid write_state arguments"); return -1; }
    Context &c = h->impl;
    if (c.cap <= 0) { set_error("no resident state"); return -1; }
    CROMA_CUDA(cudaSetDevice(c.device));
    CromaB200Output *outs[2] = {cre_out, crp_out};
    const double *src[2] = {c.d_cre, c.d_crp};
    for (int k = 0; k < 2; k++) {
        CromaB200Output *o = outs[k];
        if (!o) continue;
        int rc = check_slab(o, slab);
        if (rc) return rc;
        if (o->nrow != (size_t)c.cap || o->ncol != (size_t)NB) {
            set_error("output rows / columns differ from the context's tracers / bins");
            return -1;
        }
        rc = queue_device_slab(o, c, src[k], slab, rho_gcc, output_per_cc);
        if (rc) return rc;
    }
    return 0;
}

int croma_b200_output_flush(CromaB200Output *o)
{
    if (!o) { set_error("null output"); return -1; }
    std::unique_lock<std::mutex> lk(o->mu);
    o->cv.wait(lk, [&] { return o->pending == 0; });
    if (o->err) {
        set_error(o->err_msg);
        return o->err;
    }
    return 0;
}

int croma_b200_output_close(CromaB200Output *o)
{
    if (!o) return 0;
    int rc = croma_b200_output_flush(o);
    if (o->writer.joinable()) {
        {
            std::lock_guard<std::mutex> lk(o->mu);
            o->stop = true;
        }
        o->cv.notify_all();
        o->writer.join();
    }
    if (o->device >= 0) {
        cudaSetDevice(o->device);
        if (o->copy_stream) {
            cudaStreamSynchronize(o->copy_stream);
            cudaStreamDestroy(o->copy_stream);
        }
        cudaFree(o->d_stage);
        cudaFree(o->d_rho);
        for (int s = 0; s < 2; s++) {
            if (o->h_slot[s]) cudaFreeHost(o->h_slot[s]);
            if (o->ev_copied[s]) cudaEventDestroy(o->ev_copied[s]);
        }
        if (o->ev_staged) cudaEventDestroy(o->ev_staged);
    }
    if (o->fd >= 0) {
        if (fsync(o->fd) != 0 && !rc) rc = io_fail("fsync " + o->path);
        if (close(o->fd) != 0 && !rc) rc = io_fail("close " + o->path);
    }
    delete o;
    return rc;
}

int croma_b200_checkpoint_write_host(const CromaB200Checkpoint *ck, int np_bins, int npe_bins, const double *crp,
                                     const double *cre)
{
    int rc = check_ckpt(ck);
    if (rc) return rc;
    if (!crp || !cre || np_bins <= 0 || npe_bins <= 0) { set_error("invalid checkpoint state"); return -1; }
    if (ensure_dir(ck->dir) != 0) return io_fail(std::string("checkpoint directory ") + ck->dir);
    const std::string path = ckpt_path(ck->dir, ck->mpi_rank), tmp = path + ".tmp";
    CkptHeader hd;
    memset(&hd, 0, sizeof hd);
    snprintf(hd.magic, sizeof hd.magic, "TFPCHK1");
    hd.version = 1;
    hd.mpi_rank = ck->mpi_rank;
    hd.world_size = ck->world_size;
    hd.ntracer = ck->ntracer;
    hd.ntracer_global = ck->ntracer_global;
    hd.nsnap = ck->nsnap;
    hd.nfreq = ck->nfreq;
    hd.np_bins = np_bins;
    hd.npe_bins = npe_bins;
    hd.nsnp_i_value = ck->nsnp_i;
    hd.nsnp_f_value = ck->nsnp_f;
    hd.completed_snapshot = ck->completed_snapshot;
    hd.tracer_start = ck->tracer_start;
    FILE *fp = fopen(tmp.c_str(), "wb");
    if (!fp) return io_fail("open " + tmp);
    const size_t n = (size_t)ck->ntracer;
    bool ok = fwrite(&hd, sizeof hd, 1, fp) == 1 && fwrite(ck->tracer_ids, sizeof(int), n, fp) == n &&
              fwrite(crp, sizeof(double), n * (size_t)np_bins, fp) == n * (size_t)np_bins &&
              fwrite(cre, sizeof(double), n * (size_t)npe_bins, fp) == n * (size_t)npe_bins &&
              fflush(fp) == 0 && fsync(fileno(fp)) == 0;
    if (!ok) {
        const int e = errno;
        fclose(fp);
        errno = e;
        return io_fail("write " + tmp);
    }
    if (fclose(fp) != 0) return io_fail("close " + tmp);
    if (rename(tmp.c_str(), path.c_str()) != 0) return io_fail("rename " + tmp);
    return 0;
}

int croma_b200_checkpoint_read_host(const CromaB200Checkpoint *ck, int np_bins, int npe_bins, double *crp,
                                    double *cre, int *completed_snapshot)
{
    int rc = check_ckpt(ck);
    if (rc) return rc;
    if (!crp || !cre || !completed_snapshot) { set_error("invalid checkpoint outputs"); return -1; }
    const std::string path = ckpt_path(ck->dir, ck->mpi_rank);
    FILE *fp = fopen(path.c_str(), "rb");
    if (!fp) return io_fail("open " + path);
    CkptHeader hd;
    const size_t n = (size_t)ck->ntracer;
    std::vector<int> ids(n);
    rc = -1;
    if (fread(&hd, sizeof hd, 1, fp) != 1) {
        set_error("short checkpoint header in " + path);
    } else if (strncmp(hd.magic, "TFPCHK1", sizeof hd.magic) != 0 || hd.version != 1) {
        set_error("not a TFPCHK1 version 1 checkpoint: " + path);
    } else if (hd.mpi_rank != ck->mpi_rank || hd.world_size != ck->world_size || hd.ntracer != ck->ntracer ||
               hd.ntracer_global != ck->ntracer_global || hd.nsnap != ck->nsnap || hd.nfreq != ck->nfreq ||
               hd.np_bins != np_bins || hd.npe_bins != npe_bins || hd.nsnp_i_value != ck->nsnp_i ||
               hd.nsnp_f_value != ck->nsnp_f || hd.tracer_start != ck->tracer_start ||
               hd.completed_snapshot < 0 || hd.completed_snapshot >= ck->nsnap) {
        set_error("checkpoint metadata mismatch in " + path);
    } else if (fread(ids.data(), sizeof(int), n, fp) != n) {
        set_error("short checkpoint tracer ids in " + path);
    } else if (memcmp(ids.data(), ck->tracer_ids, n * sizeof(int)) != 0) {
        set_error("checkpoint tracer order mismatch in " + path);
    } else if (fread(crp, sizeof(double), n * (size_t)np_bins, fp) != n * (size_t)np_bins ||
               fread(cre, sizeof(double), n * (size_t)npe_bins, fp) != n * (size_t)npe_bins) {
        set_error("short checkpoint spectra in " + path);
    } else {
        *completed_snapshot = hd.completed_snapshot;
        rc = 0;
    }
    fclose(fp);
    return rc;
}

int croma_b200_checkpoint_write(CromaB200Context *h, const CromaB200Checkpoint *ck)
{
    if (!h) { set_error("null context"); return -1; }
    int rc = check_ckpt(ck);
    if (rc) return rc;
    if (ck->ntracer != h->impl.cap) { set_error("checkpoint ntracer differs from the context's"); return -1; }
    std::vector<double> crp((size_t)ck->ntracer * NB), cre((size_t)ck->ntracer * NB);
    rc = croma_b200_get_state(h, crp.data(), cre.data());
    if (rc) return rc;
    return croma_b200_checkpoint_write_host(ck, NB, NB, crp.data(), cre.data());
}

int croma_b200_checkpoint_read(CromaB200Context *h, const CromaB200Checkpoint *ck, int *completed_snapshot)
{
    if (!h) { set_error("null context"); return -1; }
    int rc = check_ckpt(ck);
    if (rc) return rc;
    std::vector<double> crp((size_t)ck->ntracer * NB), cre((size_t)ck->ntracer * NB);
    rc = croma_b200_checkpoint_read_host(ck, NB, NB, crp.data(), cre.data(), completed_snapshot);
    if (rc) return rc;
    return croma_b200_set_state(h, ck->ntracer, crp.data(), cre.data(), nullptr, nullptr, nullptr, nullptr);
}

}  // extern "C"
