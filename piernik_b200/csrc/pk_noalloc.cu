// pk_noalloc.cu -- pk_timestep_raw_noalloc: the raw CFL time step of blocks
// whose states the caller already holds in device memory, computed without
// allocating anything.
//
// Why it exists: every other entry point works through a handle, and
// pk_create / pk_block_add / pk_timestep_raw allocate device memory (the
// block buffers and the reduction slots).  Some host codes cannot allow
// that: a code that has reserved the device's memory for its own pool
// allocator, or that must not let a cudaMalloc synchronise the device in the
// middle of its step loop, can still ask for the CFL limit of the state it
// owns through this function.
//
// The reduction slots live in a fixed file-scope device array of
// PK_NOALLOC_MAX_BLOCKS x 12 words (6 KiB), which every GPU that loads the
// library holds until the process exits.  All calls share it: calls that
// overlap on a GPU (other streams, other host threads) race on it and give
// wrong results.  Each call clears the slots it uses before the reduction.
// The first call on a device looks up the array's device address with that
// device current (cudaGetSymbolAddress).  The call is synchronous (it reads
// the reduction back and waits for its stream), so it is never made while
// its stream is capturing: it checks that and returns PK_E_STATE.  The
// stream and every state must belong to the current device (PK_E_ARG
// otherwise, before anything is launched).
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/piernik_b200.h"
#include "pk_aux.cuh"

using namespace pk;

// the scratch: one row of 12 bit patterns (3 fluids x c_x, c_y, c_z, max_d c_d,
// as k_cfl writes them) per block of a call
static __device__ __align__(256) unsigned long long g_cfl_slots[12 * PK_NOALLOC_MAX_BLOCKS];

namespace {

constexpr int SLOTS = 12;
constexpr int MAX_DEVICES = 64;

std::mutex g_setup_mutex;
unsigned long long* g_slots_dev[MAX_DEVICES] = {};   // device address of g_cfl_slots per device

int say(char* err, int32_t errlen, int code, const char* msg)
{
    if (err && errlen > 0) {
        std::strncpy(err, msg, (size_t)errlen - 1);
        err[errlen - 1] = '\0';
    }
    return code;
}

// Device address of the slots on the current device; looked up once per device.
int slots_of_current_device(unsigned long long** out, char* err, int32_t errlen)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return say(err, errlen, PK_E_CUDA, "cudaGetDevice failed");
    if (dev >= MAX_DEVICES) return say(err, errlen, PK_E_UNSUPPORTED, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_slots_dev[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_cfl_slots);
        if (e != cudaSuccess || !p) {
            char msg[160];
            std::snprintf(msg, sizeof msg, "cudaGetSymbolAddress of the scratch slots failed: %s",
                          cudaGetErrorString(e));
            return say(err, errlen, PK_E_CUDA, msg);
        }
        g_slots_dev[dev] = static_cast<unsigned long long*>(p);
    }
    *out = g_slots_dev[dev];
    return PK_OK;
}

}  // namespace

extern "C" int pk_timestep_raw_noalloc(const pk_config* cfg, int32_t nblocks, const int32_t* n, const double* dl,
                                       const double* const* states, void* stream, double* dt_out,
                                       double* c_all_out, char* err, int32_t errlen)
{
    if (!cfg || !n || !dl || !states) return say(err, errlen, PK_E_ARG, "null argument");
    if (nblocks < 1) return say(err, errlen, PK_E_ARG, "nblocks must be at least 1");
    if (nblocks > PK_NOALLOC_MAX_BLOCKS) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "nblocks = %d exceeds PK_NOALLOC_MAX_BLOCKS = %d (the fixed scratch size)",
                      (int)nblocks, PK_NOALLOC_MAX_BLOCKS);
        return say(err, errlen, PK_E_ARG, msg);
    }
    if (cfg->nfluids < 1 || cfg->nfluids > 3) return say(err, errlen, PK_E_ARG, "nfluids must be 1..3");
    if (cfg->nb < 1) return say(err, errlen, PK_E_ARG, "nb must be at least 1");
    // the same fluid table as a handle builds (component planes in flind order, then B)
    CflArgs a;
    a.nfl = cfg->nfluids;
    int beg = 0;
    for (int f = 0; f < 3; ++f) {
        const int kind = f < a.nfl ? cfg->fluid_kind[f] : K_NONE;
        if (f < a.nfl && kind != PK_FLUID_ION && kind != PK_FLUID_NEU && kind != PK_FLUID_DST)
            return say(err, errlen, PK_E_ARG, "unknown fluid kind");
        a.fl[f].kind = kind;
        a.fl[f].beg = beg;
        a.fl[f].gam = (kind == PK_FLUID_DST) ? -1.0 : cfg->gamma[f];
        a.fl[f].gam_1 = a.fl[f].gam - 1.0;
        if (f < a.nfl) beg += (kind == PK_FLUID_DST) ? 4 : 5;
    }
    a.magnetic = cfg->magnetic;
    a.ib = beg;
    for (int i = 0; i < nblocks; ++i) {
        if (!states[i]) return say(err, errlen, PK_E_ARG, "null block state");
        for (int d = 0; d < 3; ++d)
            if (n[3 * i + d] < 1 || !(dl[3 * i + d] > 0.0))
                return say(err, errlen, PK_E_ARG, "block extent and cell size must be positive");
    }

    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return say(err, errlen, PK_E_CUDA, "cudaGetDevice failed");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the stream must not be capturing (the call reads its result back and
    // synchronises) and must be one of the current device's
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
        (void)cudaGetLastError();
        return say(err, errlen, PK_E_STATE, "the stream is capturing: this call synchronises and cannot be captured");
    }
    if (s) {
        int sdev = -1;
        if (cudaStreamGetDevice(s, &sdev) != cudaSuccess) {
            (void)cudaGetLastError();
            return say(err, errlen, PK_E_ARG, "invalid stream");
        }
        if (sdev != dev) return say(err, errlen, PK_E_ARG, "stream belongs to another device than the current one");
    }
    // every state must be device (or managed) memory of the current device
    for (int i = 0; i < nblocks; ++i) {
        cudaPointerAttributes pa;
        if (cudaPointerGetAttributes(&pa, states[i]) != cudaSuccess) {
            (void)cudaGetLastError();
            return say(err, errlen, PK_E_ARG, "block state is not a CUDA pointer");
        }
        if (pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged)
            return say(err, errlen, PK_E_ARG, "block state is not device memory");
        if (pa.type == cudaMemoryTypeDevice && pa.device != dev)
            return say(err, errlen, PK_E_ARG, "block state lives on another device than the current one");
    }
    int nsm = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1)
        return say(err, errlen, PK_E_CUDA, "cudaDeviceGetAttribute failed");

    unsigned long long* slots = nullptr;
    if (int rc = slots_of_current_device(&slots, err, errlen)) return rc;
    const size_t bytes = sizeof(unsigned long long) * SLOTS * (size_t)nblocks;
    // the maxima start from zero bits (below every positive double)
    if (cudaMemsetAsync(slots, 0, bytes, s) != cudaSuccess) return say(err, errlen, PK_E_CUDA, "cudaMemsetAsync failed");
    for (int i = 0; i < nblocks; ++i) {
        BoxGeom bg;
        for (int d = 0; d < 3; ++d) {
            bg.n[d] = n[3 * i + d];
            bg.g[d] = bg.n[d] > 1 ? cfg->nb : 0;
            bg.ext[d] = bg.n[d] + 2 * bg.g[d];
        }
        bg.plane = (long long)bg.ext[0] * bg.ext[1] * bg.ext[2];
        const long long ncell = (long long)bg.n[0] * bg.n[1] * bg.n[2];
        long long grid = (ncell + 255) / 256;
        if (grid > (long long)nsm * 16) grid = (long long)nsm * 16;
        k_cfl<<<(int)grid, 256, 0, s>>>(bg, states[i], a, slots + SLOTS * i);
    }
    if (cudaGetLastError() != cudaSuccess) return say(err, errlen, PK_E_CUDA, "k_cfl launch failed");
    unsigned long long h_slots[SLOTS * PK_NOALLOC_MAX_BLOCKS];
    if (cudaMemcpyAsync(h_slots, slots, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return say(err, errlen, PK_E_CUDA, "reading the reduction back failed");
    double dt = DBL_MAX, c_all = 0.0;                     // timestep.F90:161-162
    for (int i = 0; i < nblocks; ++i) {
        for (int f = 0; f < cfg->nfluids; ++f) {
            double cm[4];
            for (int d = 0; d < 4; ++d) std::memcpy(&cm[d], &h_slots[SLOTS * i + 4 * f + d], sizeof(double));
            double dtp[3];
            for (int d = 0; d < 3; ++d)
                dtp[d] = (n[3 * i + d] > 1 && cm[d] > 0.0) ? dl[3 * i + d] / cm[d] : DBL_MAX;
            double m = dtp[0];
            m = (dtp[1] < m) ? dtp[1] : m;
            m = (dtp[2] < m) ? dtp[2] : m;
            const double dtf = cfg->cfl * m;            // timestep.F90:493
            dt = (dtf < dt) ? dtf : dt;
            c_all = (cm[3] > c_all) ? cm[3] : c_all;
        }
    }
    if (dt_out) *dt_out = dt;
    if (c_all_out) *c_all_out = c_all;
    return say(err, errlen, PK_OK, "");
}
