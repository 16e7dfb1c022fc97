// Loading node tables into the resident store: the reads of exmarg/search/store.py:23-74
// (load_redshift_store's readers) and the copies of store.py:110-120 (upload) as one pipeline.
//
// A node table is nrows = ntau * nphif * nb rows of nd float32 (C order), taken either from a file
// at a byte offset (the data of the uncompressed T.npy member of a bd_*.npz) or from a host array.
// The rows are cut into chunks of whole rows.  Reader threads fill a ring of pinned host buffers
// (pread, optionally O_DIRECT with the read widened to 4 KiB boundaries, or memcpy from a host
// array); the calling thread takes the chunks in order, copies each one contiguously to a device
// staging buffer of the same ring slot, records the slot's event and re-pitches the rows into the
// table (rows padded from nd to ndp elements) with a small kernel.  A reader refills a slot only
// after its event has completed.  16-bit stores: the rows go to a float32 scratch node and the
// node is quantized on the device after its last chunk (exm_store_quantize, as exm_store_set_node).
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace {

constexpr size_t kIoAlign = 4096;   // O_DIRECT: buffer, offset and length in whole 4 KiB blocks

__global__ void __launch_bounds__(256) k_repitch(float *__restrict__ dst, int dp, const float *__restrict__ src, int sp,
                                                 int nd, long long nrows)
{
    const long long n = nrows * nd;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / nd, c = i - r * nd;
        dst[r * dp + c] = src[r * sp + c];
    }
}

struct Chunk {
    int node;
    long long row0, nrows;
};

struct Files {
    std::vector<int> fd_buf, fd_dir;
    ~Files()
    {
        for (int fd : fd_buf)
            if (fd >= 0) close(fd);
        for (int fd : fd_dir)
            if (fd >= 0) close(fd);
    }
};

struct DeviceBufs {
    exm_ctx *ctx;
    dbuf stage, scratch;
    ~DeviceBufs()
    {
        if (stage.p) exm_free(ctx, stage);
        if (scratch.p) exm_free(ctx, scratch);
    }
};

struct PinnedRing {
    char *host = nullptr;
    std::vector<cudaEvent_t> ev;
    ~PinnedRing()
    {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        if (host) cudaFreeHost(host);
    }
};

// read [a, e) of a file into buf; with O_DIRECT the read covers the enclosing 4 KiB blocks and
// *skip says where byte a landed.  Returns 0 or an errno.
int read_range(int fd, bool direct, char *buf, long long a, long long e, size_t *skip)
{
    long long a0 = a, e0 = e;
    if (direct) {
        a0 = a & ~(long long)(kIoAlign - 1);
        e0 = (e + (long long)kIoAlign - 1) & ~(long long)(kIoAlign - 1);
    }
    long long got = 0;
    const long long need = e - a0;
    while (got < need) {
        const ssize_t r = pread(fd, buf + got, (size_t)(e0 - a0 - got), a0 + got);
        if (r < 0) {
            if (errno == EINTR) continue;
            return errno;
        }
        if (r == 0) return EIO;   // end of file before the table ended
        got += r;
    }
    *skip = (size_t)(a - a0);
    return 0;
}

}   // namespace

void exm_store_load_run(exm_ctx *ctx, int first, int n, const char *const *paths, const int64_t *offsets,
                        const float *const *hosts, int readers, long long chunk_bytes, int flags, double *stats)
{
    using clk = std::chrono::steady_clock;
    const auto t_start = clk::now();
    const int nd = ctx->nd, ndp = ctx->ndp;
    const size_t rowb = sizeof(float) * (size_t)nd;
    const long long nrows = (long long)ctx->ntau * ctx->nphif * ctx->nb;
    const long long cr = std::max(1LL, std::min(nrows, (chunk_bytes > 0 ? chunk_bytes : (8LL << 20)) / (long long)rowb));
    const bool want_direct = (flags & EXM_LOAD_DIRECT) != 0;

    // the files: sizes checked before any transfer
    Files fs;
    fs.fd_buf.assign(n, -1);
    fs.fd_dir.assign(n, -1);
    int n_direct = 0;
    for (int i = 0; i < n; ++i) {
        if (!paths || !paths[i]) {
            if (!hosts || !hosts[i]) EXM_THROW(EXM_ERR_ARG, "node " + std::to_string(first + i) + ": no file and no host table");
            continue;
        }
        if (offsets[i] < 0) EXM_THROW(EXM_ERR_ARG, "negative table offset");
        fs.fd_buf[i] = open(paths[i], O_RDONLY | O_CLOEXEC);
        if (fs.fd_buf[i] < 0) EXM_THROW(EXM_ERR_ARG, std::string("cannot open ") + paths[i] + ": " + strerror(errno));
        struct stat st;
        if (fstat(fs.fd_buf[i], &st) != 0) EXM_THROW(EXM_ERR_ARG, std::string("cannot stat ") + paths[i]);
        if ((long long)st.st_size < offsets[i] + nrows * (long long)rowb)
            EXM_THROW(EXM_ERR_ARG, std::string(paths[i]) + " ends before its table does");
        if (want_direct) {
            fs.fd_dir[i] = open(paths[i], O_RDONLY | O_CLOEXEC | O_DIRECT);   // refused by some file systems
            n_direct += fs.fd_dir[i] >= 0;
        }
    }

    std::vector<Chunk> jobs;
    for (int i = 0; i < n; ++i)
        for (long long r = 0; r < nrows; r += cr) jobs.push_back({i, r, std::min(cr, nrows - r)});
    const int njobs = (int)jobs.size();
    const int nrd = std::max(1, std::min(readers, njobs));
    const int nbuf = std::max(1, std::min(njobs, 2 * nrd + 2));
    const size_t slot = ((size_t)cr * rowb + 2 * kIoAlign + kIoAlign - 1) & ~(kIoAlign - 1);

    PinnedRing ring;
    EXM_CUDA(cudaHostAlloc((void **)&ring.host, slot * nbuf, cudaHostAllocDefault));
    ring.ev.resize(nbuf);
    for (int b = 0; b < nbuf; ++b) EXM_CUDA(cudaEventCreateWithFlags(&ring.ev[b], cudaEventDisableTiming));
    DeviceBufs dv{ctx, {}, {}};
    exm_alloc(ctx, dv.stage, (size_t)cr * rowb * nbuf);
    if (ctx->dtype != EXM_DTYPE_F32) exm_alloc(ctx, dv.scratch, (size_t)nrows * rowb);

    std::mutex mu;
    std::condition_variable cv;
    std::atomic<int> next{0};
    std::vector<char> filled(njobs, 0);
    std::vector<size_t> skip(njobs, 0);
    int issued = 0;
    bool stop = false;
    std::string rd_err;
    std::atomic<long long> file_bytes{0}, host_bytes{0};
    std::atomic<long long> read_ns{0};

    auto fail = [&](const std::string &m) {
        std::lock_guard<std::mutex> lk(mu);
        if (rd_err.empty()) rd_err = m;
        stop = true;
        cv.notify_all();
    };
    auto reader = [&]() {
        cudaSetDevice(ctx->dev);
        for (;;) {
            const int j = next.fetch_add(1);
            if (j >= njobs) return;
            const int b = j % nbuf;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || issued > j - nbuf; });
                if (stop) return;
            }
            if (j >= nbuf) {
                const cudaError_t e = cudaEventSynchronize(ring.ev[b]);
                if (e != cudaSuccess) return fail(std::string("staging copy: ") + cudaGetErrorString(e));
            }
            const Chunk &c = jobs[j];
            char *buf = ring.host + (size_t)b * slot;
            const size_t len = (size_t)c.nrows * rowb;
            const auto t0 = clk::now();
            size_t sk = 0;
            if (fs.fd_buf[c.node] >= 0) {
                const long long a = offsets[c.node] + c.row0 * (long long)rowb;
                int rc = EINVAL;
                if (fs.fd_dir[c.node] >= 0) rc = read_range(fs.fd_dir[c.node], true, buf, a, a + (long long)len, &sk);
                if (rc == EINVAL) rc = read_range(fs.fd_buf[c.node], false, buf, a, a + (long long)len, &sk);
                if (rc != 0) return fail(std::string("reading ") + paths[c.node] + ": " + strerror(rc));
                file_bytes += (long long)len;
            } else {
                memcpy(buf, (const char *)hosts[c.node] + c.row0 * (long long)rowb, len);
                host_bytes += (long long)len;
            }
            read_ns += std::chrono::duration_cast<std::chrono::nanoseconds>(clk::now() - t0).count();
            {
                std::lock_guard<std::mutex> lk(mu);
                skip[j] = sk;
                filled[j] = 1;
            }
            cv.notify_all();
        }
    };

    std::vector<std::thread> pool;
    long long wait_ns = 0;
    std::string iss_err;
    int iss_code = 0;
    try {
        for (int t = 0; t < nrd; ++t) pool.emplace_back(reader);
    } catch (const std::exception &e) {   // a reader could not start: stop the ones that did
        iss_code = EXM_ERR_STATE;
        iss_err = std::string("store load: cannot start reader threads: ") + e.what();
    }
    try {
        for (int j = 0; j < njobs && iss_code == 0; ++j) {   // (no issue at all when a reader did not start)
            const auto t0 = clk::now();
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || filled[j]; });
                if (stop) break;
            }
            wait_ns += std::chrono::duration_cast<std::chrono::nanoseconds>(clk::now() - t0).count();
            const Chunk &c = jobs[j];
            const int b = j % nbuf;
            const size_t len = (size_t)c.nrows * rowb;
            float *st = (float *)dv.stage.p + (size_t)b * cr * nd;
            EXM_CUDA(cudaMemcpyAsync(st, ring.host + (size_t)b * slot + skip[j], len, cudaMemcpyHostToDevice, ctx->stream));
            EXM_CUDA(cudaEventRecord(ring.ev[b], ctx->stream));
            const int k = first + c.node;
            float *dst;
            int dp;
            if (ctx->dtype == EXM_DTYPE_F32) {
                dst = (float *)ctx->T.p + (size_t)k * ctx->tstride + (size_t)c.row0 * ndp;
                dp = ndp;
            } else {
                dst = (float *)dv.scratch.p + (size_t)c.row0 * nd;
                dp = nd;
            }
            const long long nel = c.nrows * nd;
            const int grid = (int)std::min<long long>((nel + 255) / 256, (long long)ctx->sm_count * 8);
            k_repitch<<<grid, 256, 0, ctx->stream>>>(dst, dp, st, nd, nd, c.nrows);
            EXM_CUDA(cudaGetLastError());
            if (ctx->dtype != EXM_DTYPE_F32 && c.row0 + c.nrows == nrows) exm_store_quantize(ctx, k, (const float *)dv.scratch.p, nd);
            {
                std::lock_guard<std::mutex> lk(mu);
                issued = j + 1;
            }
            cv.notify_all();
        }
    } catch (const exm_error &e) {
        iss_code = e.code;
        iss_err = e.msg;
    } catch (const std::bad_alloc &) {
        iss_code = EXM_ERR_OOM;
        iss_err = "store load: host memory exhausted";
    } catch (const std::exception &e) {
        iss_code = EXM_ERR_CUDA;
        iss_err = std::string("store load: ") + e.what();
    }
    {
        std::lock_guard<std::mutex> lk(mu);
        if (iss_code) stop = true;
    }
    cv.notify_all();
    for (auto &t : pool) t.join();
    const cudaError_t se = cudaStreamSynchronize(ctx->stream);
    if (iss_code) throw exm_error{iss_code, iss_err};
    if (!rd_err.empty()) EXM_THROW(EXM_ERR_ARG, rd_err);
    if (se != cudaSuccess) EXM_THROW(EXM_ERR_CUDA, std::string("store load: ") + cudaGetErrorString(se));
    if (stats) {
        stats[0] = std::chrono::duration<double>(clk::now() - t_start).count();
        stats[1] = (double)file_bytes.load();
        stats[2] = (double)host_bytes.load();
        stats[3] = (double)n_direct;
        stats[4] = (double)nbuf;
        stats[5] = (double)(cr * (long long)rowb);
        stats[6] = (double)read_ns.load() * 1e-9;
        stats[7] = (double)wait_ns * 1e-9;
    }
}
