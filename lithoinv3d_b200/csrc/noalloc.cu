// lf_forward_noalloc: the single-body gz + TMI forward for callers that
// cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is unavailable or forbidden --
// inside a host framework that owns every device allocation through its own
// pool, in a process whose memory budget is fixed up front, or in a plugin
// called from a real-time loop that must not allocate.  Such callers already
// hold their inputs and outputs in device memory and pass those pointers in.
//
// What it uses instead of allocations: one file-scope __device__ scratch array
// of kNoallocScratchBytes (8 MiB).  Every GPU that loads this library holds it
// until the process exits.  The library looks up its device address once per
// device with cudaGetSymbolAddress, on the first call made on that device, and
// keeps it for the life of the process: a cudaDeviceReset of that device
// invalidates the kept address, so calling this entry point after a device
// reset is not supported.  All calls share the array and every call
// overwrites the regions it reads (nothing in it has to start at zero), except
// the error flag, which each call clears first; calls that overlap on the GPU
// (two streams, two threads) race on it: serialise them.
//
// Every call reads its error flag back into host memory and waits for its
// stream, neither of which is legal while the stream is being captured into a
// CUDA graph: the entry point refuses a capturing stream (LF_EINVAL) instead of
// invalidating the caller's capture.  An error already pending on the calling
// thread when the call starts (a failed launch of the caller's own) is left in
// place and reported as LF_ECUDA before any work is queued.
//
// The kernels are the library's FP64 forward (facet constants, station-tiled
// pair kernel, chunk reduction) specialised to one group.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

#include "../../include/litho_gpu.h"

namespace {
#include "kernels_fp64.cuh"
}  // namespace

namespace {

constexpr size_t kNoallocScratchBytes = size_t(8) << 20;
constexpr size_t kNoallocScratchDoubles = kNoallocScratchBytes / sizeof(double);
constexpr int kMaxDevices = 64;

// The only scratch this entry point uses.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

std::mutex g_mutex;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on `dev` (looked up once per device,
// with that device current).
cudaError_t scratch_address(int dev, double** out) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = p;
    }
    *out = static_cast<double*>(g_scratch_addr[dev]);
    return cudaSuccess;
}

struct SingleGroup {
    double gscale;  // G * rho * 1e3 * 1e5
    double mscale;  // amp * 100 / (4 pi)
    litho_b200::d3 mdir, fdir;
};

// Facet constants of one group; triangle indices are bounds-checked against
// nv (a bad facet is marked invalid and raises the error flag).
__global__ void k_na_prep(int nv, const double* __restrict__ xyz, int nt, const int32_t* __restrict__ tri,
                          SingleGroup g, double* __restrict__ fc, int* __restrict__ err) {
    using namespace litho_b200;
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nt) return;
    int ia = tri[3 * f], ib = tri[3 * f + 1], ic = tri[3 * f + 2];
    double out[NFC];
    for (int k = 0; k < NFC; ++k) out[k] = 0.0;
    if (ia < 0 || ia >= nv || ib < 0 || ib >= nv || ic < 0 || ic >= nv) {
        atomicExch(err, 1);
    } else {
        d3 v[3] = {mk3(xyz[3 * ia], xyz[3 * ia + 1], xyz[3 * ia + 2]), mk3(xyz[3 * ib], xyz[3 * ib + 1], xyz[3 * ib + 2]),
                   mk3(xyz[3 * ic], xyz[3 * ic + 1], xyz[3 * ic + 2])};
        d3 n = cross_rn(sub_rn(v[1], v[0]), sub_rn(v[2], v[0]));
        double area2 = norm_rn(n);
        bool valid = !(area2 < kEps);
        d3 un = valid ? div_rn(n, area2) : mk3(0, 0, 0);
        out[FC_AX] = v[0].x; out[FC_AY] = v[0].y; out[FC_AZ] = v[0].z;
        out[FC_BX] = v[1].x; out[FC_BY] = v[1].y; out[FC_BZ] = v[1].z;
        out[FC_CX] = v[2].x; out[FC_CY] = v[2].y; out[FC_CZ] = v[2].z;
        out[FC_NX] = un.x; out[FC_NY] = un.y; out[FC_NZ] = un.z;
        out[FC_MF] = __dmul_rn(dot_rn(g.mdir, un), dot_rn(g.fdir, un));
        for (int i = 0; i < 3; ++i) {
            d3 e = sub_rn(v[(i + 1) % 3], v[i]);
            double L = norm_rn(e);
            d3 eh = (L < kEps) ? mk3(0, 0, 0) : div_rn(e, L);
            d3 perp = cross_rn(un, eh);
            out[FC_E0X + 3 * i] = e.x; out[FC_E0Y + 3 * i] = e.y; out[FC_E0Z + 3 * i] = e.z;
            out[FC_L0 + i] = L;
            out[FC_P0X + 3 * i] = perp.x; out[FC_P0Y + 3 * i] = perp.y; out[FC_P0Z + 3 * i] = perp.z;
            out[FC_MT0 + i] = __dmul_rn(dot_rn(g.mdir, perp), dot_rn(g.fdir, perp));
        }
        out[FC_VALID] = valid ? 1.0 : 0.0;
    }
    for (int k = 0; k < NFC; ++k) fc[(size_t)k * nt + f] = out[k];
}

// Station-tiled pair kernel over uniform facet chunks of `cs` facets.
template <int FT>
__global__ void __launch_bounds__(128) k_na_forward(int ns, const double* __restrict__ sta, int nt, int cs,
                                                    const double* __restrict__ fc, double* __restrict__ part_gz,
                                                    double* __restrict__ part_tmi) {
    using namespace litho_b200;
    __shared__ double sm[NFC * FT];
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    int chunk = blockIdx.y;
    int fb = chunk * cs, fe = min(nt, fb + cs);
    d3 o = mk3(0, 0, 0);
    if (s < ns) o = mk3(sta[3 * s], sta[3 * s + 1], sta[3 * s + 2]);
    double gz = 0.0, tmi = 0.0;
    for (int f0 = fb; f0 < fe; f0 += FT) {
        int nf = min(FT, fe - f0);
        __syncthreads();
        for (int idx = threadIdx.x; idx < NFC * FT; idx += blockDim.x) {
            int k = idx / FT, j = idx % FT;
            sm[idx] = (j < nf) ? fc[(size_t)k * nt + f0 + j] : 0.0;
        }
        __syncthreads();
        if (s < ns)
            for (int j = 0; j < nf; ++j) pair_forward_fp64<true, true>(sm, j, FT, o, &gz, &tmi);
    }
    if (s < ns) {
        part_gz[(size_t)chunk * ns + s] = gz;
        part_tmi[(size_t)chunk * ns + s] = tmi;
    }
}

__global__ void k_na_reduce(int ns, int nch, const double* __restrict__ part_gz, const double* __restrict__ part_tmi,
                            SingleGroup g, double* __restrict__ gz, double* __restrict__ tmi) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    double tg = 0.0, tt = 0.0;
    for (int c = 0; c < nch; ++c) {
        tg += part_gz[(size_t)c * ns + s];
        tt += part_tmi[(size_t)c * ns + s];
    }
    if (gz) gz[s] = tg * g.gscale;
    if (tmi) tmi[s] = -g.mscale * tt;
}

}  // namespace

extern "C" lf_status lf_forward_noalloc(int nv, const double* d_xyz, int nt, const int32_t* d_tri, int ns,
                                        const double* d_sta, double density_gcc, double susceptibility_si,
                                        double inc_deg, double dec_deg, double field_nt, double* d_gz,
                                        double* d_tmi, void* stream) {
    if (nv < 3 || nt < 1 || ns < 1 || !d_xyz || !d_tri || !d_sta || (!d_gz && !d_tmi)) return LF_EINVAL;
    if (!std::isfinite(density_gcc) || !std::isfinite(susceptibility_si) || !std::isfinite(inc_deg) ||
        !std::isfinite(dec_deg) || !std::isfinite(field_nt))
        return LF_EINVAL;
    // Scratch layout (doubles): [0, 32) error flag and padding, facet constants
    // NFC * nt, then gz and TMI chunk partials 2 * nch * ns.
    const size_t head = 32;
    const size_t fcSize = (size_t)litho_b200::NFC * nt;
    if (head + fcSize + 2 * (size_t)ns > kNoallocScratchDoubles) return LF_EINVAL;
    const size_t room = (kNoallocScratchDoubles - head - fcSize) / (2 * (size_t)ns);
    int sBlocks = (ns + 127) / 128;
    int wantChunks = (148 * 4 + sBlocks - 1) / sBlocks;
    int cs = (nt + wantChunks - 1) / wantChunks;
    if (cs < 64) cs = 64;
    int nch = (nt + cs - 1) / cs;
    if ((size_t)nch > room) {
        nch = static_cast<int>(room);
        cs = (nt + nch - 1) / nch;
        nch = (nt + cs - 1) / cs;
    }
    // An error left pending by earlier work of the caller is theirs: report it
    // without clearing it, before queueing anything.
    if (cudaPeekAtLastError() != cudaSuccess) return LF_ECUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) return LF_ECUDA;
    if (cap != cudaStreamCaptureStatusNone) return LF_EINVAL;  // host read-back and sync cannot be captured
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return LF_ECUDA;
    double* base = nullptr;
    if (scratch_address(dev, &base) != cudaSuccess) return LF_ECUDA;
    int* err = reinterpret_cast<int*>(base);
    double* fc = base + head;
    double* partG = fc + fcSize;
    double* partM = partG + (size_t)nch * ns;

    // magnetisation and scales as MagneticForward / GravityForward build them
    const double pi = litho_b200::kPi;
    double I = inc_deg * pi / 180.0, D = dec_deg * pi / 180.0, cI = std::cos(I);
    SingleGroup g;
    g.fdir = {cI * std::cos(D), cI * std::sin(D), -std::sin(I)};
    double amp = std::fabs(susceptibility_si * field_nt / 100.0);
    g.mdir = (susceptibility_si * field_nt / 100.0 < 0.0) ? litho_b200::d3{-g.fdir.x, -g.fdir.y, -g.fdir.z} : g.fdir;
    if (amp < litho_b200::kEps) g.mdir = g.fdir;
    g.mscale = amp * 100.0 / (4.0 * pi);
    g.gscale = 6.67430e-11 * density_gcc * 1000.0 * 1e5;

    if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) return LF_ECUDA;
    k_na_prep<<<(nt + 127) / 128, 128, 0, st>>>(nv, d_xyz, nt, d_tri, g, fc, err);
    dim3 grid(sBlocks, nch);
    k_na_forward<32><<<grid, 128, 0, st>>>(ns, d_sta, nt, cs, fc, partG, partM);
    k_na_reduce<<<(ns + 255) / 256, 256, 0, st>>>(ns, nch, partG, partM, g, d_gz, d_tmi);
    if (cudaGetLastError() != cudaSuccess) return LF_ECUDA;
    int hErr = 0;
    if (cudaMemcpyAsync(&hErr, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return LF_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return LF_ECUDA;
    return hErr ? LF_EINVAL : LF_OK;
}
