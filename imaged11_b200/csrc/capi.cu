// C ABI, layer 1: the reference's own C signatures with host pointers.
//
// Each call stages its inputs into device memory on the calling thread's
// per-thread default stream (buffers kept per thread and device for calls up
// to 64 MB, the stream-ordered pool above that), runs the device entry point
// and copies the results back before it returns.  Calls made from different
// host threads use different streams and do not share buffers.
#include <string.h>

#include "common.cuh"

static thread_local int t_last_status = ID11B_OK;
static thread_local int t_last_cuda = 0;

namespace {
__global__ void k_fixsum_finish(double* __restrict__ sums, int64_t n, double inv_scale) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long q = reinterpret_cast<unsigned long long*>(sums)[i];
        sums[i] = (double)q * inv_scale;
    }
}
}  // namespace

int id11b_fixsum_finish(double* sums, int64_t n, double scale, cudaStream_t st) {
    if (!sums || n <= 0) return ID11B_OK;
    const int64_t blocks = (n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096;
    k_fixsum_finish<<<(unsigned)blocks, 256, 0, st>>>(sums, n, 1.0 / scale);
    ID11B_CHECK_LAUNCH();
    return ID11B_OK;
}

int id11b_record_cuda(cudaError_t e) {
    t_last_cuda = (int)e;
    return ID11B_ERR_CUDA;
}

extern "C" int id11b_version(void) { return 100; }

extern "C" const char* id11b_status_string(int status) {
    switch (status) {
        case ID11B_OK: return "ok";
        case ID11B_ERR_ARG: return "invalid argument";
        case ID11B_ERR_CUDA: return "CUDA error";
        case ID11B_ERR_ALIGN: return "misaligned pointer";
        case ID11B_ERR_SIZE: return "size beyond the supported maximum";
        case ID11B_ERR_TIMEOUT: return "bounded device wait timed out";
        case ID11B_ERR_NODEV: return "no CUDA device";
        default: return "unknown status";
    }
}

extern "C" int id11b_last_cuda_error(void) { return t_last_cuda; }
extern "C" int id11b_last_status(void) { return t_last_status; }

namespace {

// Calls of up to kKeepBytes stage through buffers kept per host thread and
// device: a device buffer and a pinned host mirror of it, grown when a call
// needs more.  Inputs are copied into the mirror and sent by DMA; outputs come
// back into the mirror and are copied out after the call's one
// synchronisation.  A small call then costs its launches and one round trip,
// not an allocation and a pageable copy per array.  Larger calls draw one
// allocation from the stream-ordered pool and copy pageable memory directly.
constexpr size_t kKeepBytes = size_t(64) << 20;
constexpr int kMaxDev = 64;

struct ThreadBufs {
    char* dev = nullptr;
    char* pin = nullptr;
    size_t cap = 0;
    ~ThreadBufs() {  // at thread exit (the runtime may already be shutting down)
        if (dev) cudaFree(dev);
        if (pin) cudaFreeHost(pin);
    }
};
thread_local ThreadBufs t_bufs[kMaxDev];
thread_local int t_ndev = -1;

struct Staging {
    cudaStream_t st = cudaStreamPerThread;
    char* base = nullptr;
    char* pin = nullptr;  // mirror of base (kept buffers), else null
    bool pooled = false;
    size_t used = 0, cap = 0;
    int status = ID11B_OK;
    struct Out {
        void* h;
        size_t off, bytes;
    };
    static constexpr int kMaxOut = 8;
    Out outs[kMaxOut];
    int nout = 0;
    explicit Staging(size_t bytes) {
        if (t_ndev < 0) {
            int nd = 0;
            if (cudaGetDeviceCount(&nd) != cudaSuccess) {
                cudaGetLastError();
                nd = 0;
            }
            t_ndev = nd;
        }
        if (t_ndev == 0) {
            status = ID11B_ERR_NODEV;
            return;
        }
        cap = bytes + 256 * 8;
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) {
            status = id11b_record_cuda(e);
            return;
        }
        if (cap <= kKeepBytes && dev < kMaxDev) {
            ThreadBufs& tb = t_bufs[dev];
            if (tb.cap < cap) {
                size_t want = tb.cap * 2 > cap ? tb.cap * 2 : cap;
                want = want < (size_t(1) << 20) ? (size_t(1) << 20) : want;
                want = want > kKeepBytes ? kKeepBytes : want;
                if (tb.dev) cudaFree(tb.dev);
                if (tb.pin) cudaFreeHost(tb.pin);
                tb.dev = tb.pin = nullptr;
                tb.cap = 0;
                e = cudaMalloc((void**)&tb.dev, want);
                if (e == cudaSuccess) e = cudaMallocHost((void**)&tb.pin, want);
                if (e != cudaSuccess) {
                    if (tb.dev) cudaFree(tb.dev);
                    tb.dev = tb.pin = nullptr;
                    status = id11b_record_cuda(e);
                    return;
                }
                tb.cap = want;
            }
            base = tb.dev;
            pin = tb.pin;
            return;
        }
        e = cudaMallocAsync((void**)&base, cap, st);
        if (e != cudaSuccess) {
            base = nullptr;
            status = id11b_record_cuda(e);
            return;
        }
        pooled = true;
    }
    ~Staging() {
        if (pooled && base) cudaFreeAsync(base, st);
    }
    template <class T>
    T* take(size_t count) {
        size_t off = (used + 255) & ~(size_t)255;
        used = off + count * sizeof(T);
        return reinterpret_cast<T*>(base + off);
    }
    int h2d(void* d, const void* h, size_t bytes) {
        if (status || !bytes) return status;
        cudaError_t e;
        if (pin) {
            const size_t off = (size_t)((char*)d - base);
            memcpy(pin + off, h, bytes);
            e = cudaMemcpyAsync(d, pin + off, bytes, cudaMemcpyHostToDevice, st);
        } else {
            e = cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st);
        }
        if (e != cudaSuccess) status = id11b_record_cuda(e);
        return status;
    }
    // put: copy into the pinned mirror now, send with the call's other inputs
    // in one DMA over the range they span (send); without a mirror, copy now
    size_t plo = ~(size_t)0, phi = 0;
    int put(void* d, const void* h, size_t bytes) {
        if (status || !bytes) return status;
        if (!pin) return h2d(d, h, bytes);
        const size_t off = (size_t)((char*)d - base);
        memcpy(pin + off, h, bytes);
        plo = off < plo ? off : plo;
        phi = off + bytes > phi ? off + bytes : phi;
        return status;
    }
    int send() {
        if (status || phi == 0) return status;
        cudaError_t e =
            cudaMemcpyAsync(base + plo, pin + plo, phi - plo, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) status = id11b_record_cuda(e);
        plo = ~(size_t)0;
        phi = 0;
        return status;
    }
    int d2h(void* h, const void* d, size_t bytes) {
        if (status || !bytes) return status;
        cudaError_t e;
        if (pin && nout < kMaxOut) {
            const size_t off = (size_t)((const char*)d - base);
            e = cudaMemcpyAsync(pin + off, d, bytes, cudaMemcpyDeviceToHost, st);
            outs[nout++] = Out{h, off, bytes};
        } else {
            e = cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st);
        }
        if (e != cudaSuccess) status = id11b_record_cuda(e);
        return status;
    }
    int run(int rc) {
        if (!status && rc) status = rc;
        return status;
    }
    int sync() {
        if (status == ID11B_ERR_NODEV) return status;
        // always drained, so that the kept buffers are idle when the call
        // returns, whatever went wrong before
        cudaError_t e = cudaStreamSynchronize(st);
        if (status) return status;
        if (e != cudaSuccess) {
            status = id11b_record_cuda(e);
            return status;
        }
        for (int i = 0; i < nout; i++) memcpy(outs[i].h, pin + outs[i].off, outs[i].bytes);
        return status;
    }
};

int finish(Staging& s) {
    s.sync();
    t_last_status = s.status;
    return s.status;
}

// The refined UBI, n and mean of one least-squares call, returned in one copy.
struct LsqResult {
    double u[9];
    double mean;
    int32_t n;
    int32_t pad;
};

}  // namespace

extern "C" void id11b_compute_gv(double xlylzl[][3], double omega[], double omegasign,
                                 double wvln, double wedge, double chi, double t[3],
                                 double gv[][3], int n) {
    if (n < 0) { t_last_status = ID11B_ERR_ARG; return; }
    Staging s(sizeof(double) * (size_t)n * 7);
    double* dx = s.take<double>(3 * (size_t)n);
    double* dom = s.take<double>(n);
    double* dg = s.take<double>(3 * (size_t)n);
    s.put(dx, xlylzl, sizeof(double) * 3 * (size_t)n);
    s.put(dom, omega, sizeof(double) * (size_t)n);
    s.send();
    if (!s.status)
        s.run(id11b_dev_compute_gv(dx, dom, omegasign, wvln, wedge, chi, t, dg, nullptr, n, s.st));
    s.d2h(gv, dg, sizeof(double) * 3 * (size_t)n);
    finish(s);
}

extern "C" void id11b_compute_geometry(double xlylzl[][3], double omega[], double omegasign,
                                       double wvln, double wedge, double chi, double t[3],
                                       double out[][6], int n) {
    if (n < 0) { t_last_status = ID11B_ERR_ARG; return; }
    Staging s(sizeof(double) * (size_t)n * 10);
    double* dx = s.take<double>(3 * (size_t)n);
    double* dom = s.take<double>(n);
    double* dout = s.take<double>(6 * (size_t)n);
    s.put(dx, xlylzl, sizeof(double) * 3 * (size_t)n);
    s.put(dom, omega, sizeof(double) * (size_t)n);
    s.send();
    if (!s.status)
        s.run(id11b_dev_compute_geometry(dx, dom, omegasign, wvln, wedge, chi, t, dout, n, s.st));
    s.d2h(out, dout, sizeof(double) * 6 * (size_t)n);
    finish(s);
}

extern "C" void id11b_compute_xlylzl(double sl[], double f[], double p[4], double r[9],
                                     double dist[3], double xlylzl[][3], int n) {
    if (n < 0) { t_last_status = ID11B_ERR_ARG; return; }
    Staging s(sizeof(double) * (size_t)n * 5);
    double* ds = s.take<double>(n);
    double* df = s.take<double>(n);
    double* dx = s.take<double>(3 * (size_t)n);
    s.put(ds, sl, sizeof(double) * (size_t)n);
    s.put(df, f, sizeof(double) * (size_t)n);
    s.send();
    if (!s.status) s.run(id11b_dev_compute_xlylzl(ds, df, p, r, dist, dx, n, s.st));
    s.d2h(xlylzl, dx, sizeof(double) * 3 * (size_t)n);
    finish(s);
}

extern "C" int id11b_score(double ubi[3][3], double gv[][3], double tol, int ng) {
    if (ng < 0) { t_last_status = ID11B_ERR_ARG; return -1; }
    Staging s(sizeof(double) * (3 * (size_t)ng + 9) + 64);
    double* du = s.take<double>(9);
    double* dg = s.take<double>(3 * (size_t)ng);
    int32_t* dc = s.take<int32_t>(1);
    int32_t count = -1;
    s.put(du, ubi, sizeof(double) * 9);
    s.put(dg, gv, sizeof(double) * 3 * (size_t)ng);
    s.send();
    if (!s.status) s.run(id11b_dev_score(du, dg, tol, ng, dc, s.st));
    s.d2h(&count, dc, sizeof(int32_t));
    return finish(s) ? -1 : count;
}

static void lsq_host(int mode, double ubi[3][3], double gv[][3], double tol, int labels[],
                     int label, int* n_out, double* mean_out, int ng) {
    if (ng < 0) { t_last_status = ID11B_ERR_ARG; return; }
    int64_t wsb = id11b_lsq_workspace_bytes(ng);
    Staging s(sizeof(double) * 3 * (size_t)ng + sizeof(LsqResult) +
              sizeof(int) * (size_t)(mode ? ng : 0) + (size_t)wsb + 64);
    LsqResult* dr = s.take<LsqResult>(1);  // UBI, then n and mean next to it
    double* dg = s.take<double>(3 * (size_t)ng);
    int32_t* dl = mode ? s.take<int32_t>(ng) : nullptr;
    char* ws = s.take<char>(wsb);
    s.put(dr->u, ubi, sizeof(double) * 9);
    s.put(dg, gv, sizeof(double) * 3 * (size_t)ng);
    if (mode) s.put(dl, labels, sizeof(int32_t) * (size_t)ng);
    s.send();
    if (!s.status) {
        if (mode == 0)
            s.run(id11b_dev_score_and_refine(dr->u, dg, tol, ng, &dr->n, &dr->mean, ws, wsb,
                                             s.st));
        else
            s.run(id11b_dev_refine_assigned(dr->u, dg, dl, label, ng, &dr->n, &dr->mean, ws, wsb,
                                            s.st));
    }
    LsqResult hr;
    s.d2h(&hr, dr, sizeof(LsqResult));
    if (finish(s) == ID11B_OK) {
        memcpy(ubi, hr.u, sizeof(hr.u));
        *n_out = hr.n;
        *mean_out = hr.mean;
    }
}

extern "C" void id11b_score_and_refine(double ubi[3][3], double gv[][3], double tol,
                                       int* n_arg, double* sumdrlv2_arg, int ng) {
    lsq_host(0, ubi, gv, tol, nullptr, 0, n_arg, sumdrlv2_arg, ng);
}

extern "C" void id11b_refine_assigned(double ubi[3][3], double gv[][3], int labels[],
                                      int label, int* npk, double* sumdrlv2, int ng) {
    lsq_host(1, ubi, gv, 0., labels, label, npk, sumdrlv2, ng);
}

extern "C" int id11b_score_and_assign(double ubi[3][3], double gv[][3], double tol,
                                      double drlv2[], int labels[], int label, int ng) {
    if (ng < 0) { t_last_status = ID11B_ERR_ARG; return -1; }
    Staging s(sizeof(double) * (4 * (size_t)ng + 9) + sizeof(int) * (size_t)ng + 64);
    double* du = s.take<double>(9);
    double* dg = s.take<double>(3 * (size_t)ng);
    double* dd = s.take<double>(ng);
    int32_t* dl = s.take<int32_t>(ng);
    int32_t* dc = s.take<int32_t>(1);
    s.put(du, ubi, sizeof(double) * 9);
    s.put(dg, gv, sizeof(double) * 3 * (size_t)ng);
    s.put(dd, drlv2, sizeof(double) * (size_t)ng);
    s.put(dl, labels, sizeof(int32_t) * (size_t)ng);
    s.send();
    if (!s.status) s.run(id11b_dev_score_and_assign(du, dg, tol, dd, dl, label, ng, dc, s.st));
    int32_t count = -1;
    s.d2h(drlv2, dd, sizeof(double) * (size_t)ng);
    s.d2h(labels, dl, sizeof(int32_t) * (size_t)ng);
    s.d2h(&count, dc, sizeof(int32_t));
    return finish(s) ? -1 : count;
}

extern "C" int id11b_verify_rounding(int n) {
    Staging s(64);
    int32_t* db = s.take<int32_t>(1);
    if (!s.status) s.run(id11b_dev_verify_rounding(n, db, s.st));
    int32_t bad = -1;
    s.d2h(&bad, db, sizeof(int32_t));
    return finish(s) ? -1 : bad;
}
