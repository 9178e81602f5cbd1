// hk_noalloc.cu -- hk_render_noalloc: the trace + shadow + shade pipeline for
// callers that must not (or cannot) allocate device memory.
//
// Who needs it: hosts that own every device allocation themselves -- a render
// plugin running inside an application with its own pooled allocator, code
// that runs while another component holds a CUDA graph capture open, or a
// process whose memory budget forbids the library from growing it. Those
// callers pass their own device buffers for the tree, the triangle records and
// the output image; everything else the pipeline needs lives in one fixed
// scratch array that is part of this library's image.
//
// The scratch array is a file-scope __device__ variable of
// HK_NOALLOC_SCRATCH_BYTES (24 MiB). Every GPU on which the library is loaded
// holds it until the process exits. All calls share it and it keeps the last
// call's contents, so the counters that must start at zero are cleared at the
// start of every call, and two calls whose GPU work overlaps (different
// streams, or different host threads on one device) race on it.
//
// Host code cannot use the array's name as a device address (it is a host-side
// stand-in), so the first call on each device looks the address up with
// cudaGetSymbolAddress while that device is current and caches it. The same
// first call also loads every kernel the entry point can launch (all accepted
// traversal variants, closest-hit and occlusion, and the ray / shading
// kernels): with lazy module loading the driver would otherwise allocate
// module memory when a variant is first launched, possibly while another
// component's stream capture is open. Make that first call before any stream
// capture begins. No cudaMalloc, cudaFree or allocating library routine is
// called.
#include <cstring>
#include <mutex>

#include "hk_common.cuh"
#include "hk_internal.h"

namespace {

constexpr size_t kScratchBytes = HK_NOALLOC_SCRATCH_BYTES;
constexpr size_t kAlign = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
unsigned char *g_scratch_dev[kMaxDevices] = {nullptr};
int g_sm_count[kMaxDevices] = {0};

size_t up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

struct Layout {
    size_t control, box, cam, lights, rays, hits, srays, shits, slot, spix, total;
};

// control block: [0] ray-batch counter, [1] error word, [2] shadow-ray count,
// [4..9] per-trace counters (unused: counting is off)
Layout layout(uint64_t npix, uint64_t nl, uint64_t npoint) {
    Layout L;
    size_t o = 0;
    L.control = o; o = up(o + 64);
    L.box = o; o = up(o + 32);
    L.cam = o; o = up(o + 64);
    L.lights = o; o = up(o + 64 * 32);
    uint64_t ns = npix * npoint;
    L.rays = o; o = up(o + npix * 32);
    L.hits = o; o = up(o + npix * 8);
    L.srays = o; o = up(o + ns * 32);
    L.shits = o; o = up(o + ns * 8);
    L.slot = o; o = up(o + npix * (nl ? nl : 1) * 4);
    L.spix = o; o = up(o + ns * 4);
    L.total = o;
    return L;
}

hk_status device_scratch(unsigned char **out, int *sm) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return HK_E_CUDA;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_dev[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return HK_E_CUDA;
        const int variants[] = {HK_TRACE_FULLSTACK, HK_TRACE_SHORTSTACK, HK_TRACE_SMEMSTACK,
                                HK_TRACE_RESTART,   HK_TRACE_RESTART_EARLY, HK_TRACE_BRUTE};
        for (int v : variants)
            if (hk::preload_trace_kernels(v) != cudaSuccess) return HK_E_CUDA;
        if (hk::preload_render_kernels() != cudaSuccess) return HK_E_CUDA;
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return HK_E_CUDA;
        g_scratch_dev[dev] = static_cast<unsigned char *>(p);
        g_sm_count[dev] = n;
    }
    *out = g_scratch_dev[dev];
    *sm = g_sm_count[dev];
    return HK_OK;
}

}  // namespace

extern "C" hk_status hk_render_noalloc(const uint32_t *d_nodes2, const uint32_t *d_refs, const float *d_records16,
                                       uint32_t ntris, const float *box8, const float *cam16,
                                       const float *lights8, uint32_t nl, uint32_t w, uint32_t h,
                                       hk_variant variant, uint32_t *d_rgba, void *cuda_stream) {
    using namespace hk;
    if (!d_nodes2 || !d_refs || !d_records16 || !box8 || !cam16 || !d_rgba || (nl && !lights8))
        return HK_E_ILLEGAL_INPUT;
    if ((reinterpret_cast<uintptr_t>(d_nodes2) & 7u) || (reinterpret_cast<uintptr_t>(d_records16) & 15u) ||
        (reinterpret_cast<uintptr_t>(d_refs) & 3u) || (reinterpret_cast<uintptr_t>(d_rgba) & 3u))
        return HK_E_ILLEGAL_INPUT;
    if ((int)variant < HK_TRACE_FULLSTACK || (int)variant > HK_TRACE_BRUTE || variant == HK_TRACE_ROPES)
        return HK_E_ILLEGAL_INPUT;
    if (nl > 64 || w == 0 || h == 0 || ntris == 0) return HK_E_ILLEGAL_INPUT;
    uint64_t npix = (uint64_t)w * h;
    uint64_t npoint = 0;
    for (uint32_t l = 0; l < nl; l++) npoint += lights8[8 * l + 3] == 1.0f;
    Layout Lo = layout(npix, nl, npoint);
    if (npix > (1u << 28) || Lo.total > kScratchBytes) return HK_E_CAPACITY;

    unsigned char *S = nullptr;
    int sm = 0;
    hk_status st = device_scratch(&S, &sm);
    if (st != HK_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    uint32_t *control = reinterpret_cast<uint32_t *>(S + Lo.control);
    float *box = reinterpret_cast<float *>(S + Lo.box);
    float *cam = reinterpret_cast<float *>(S + Lo.cam);
    float *lights = reinterpret_cast<float *>(S + Lo.lights);
    float4 *rays = reinterpret_cast<float4 *>(S + Lo.rays);
    hk_hit *hits = reinterpret_cast<hk_hit *>(S + Lo.hits);
    float4 *srays = reinterpret_cast<float4 *>(S + Lo.srays);
    hk_hit *shits = reinterpret_cast<hk_hit *>(S + Lo.shits);
    uint32_t *slot = reinterpret_cast<uint32_t *>(S + Lo.slot);
    uint32_t *spix = reinterpret_cast<uint32_t *>(S + Lo.spix);

#define HK_TRY(x)                                   \
    do {                                            \
        if ((x) != cudaSuccess) return HK_E_CUDA;   \
    } while (0)
    // the previous call's contents stay in the array: clear the counters
    HK_TRY(cudaMemsetAsync(control, 0, 64, s));
    HK_TRY(cudaMemcpyAsync(box, box8, 32, cudaMemcpyHostToDevice, s));
    HK_TRY(cudaMemcpyAsync(cam, cam16, 64, cudaMemcpyHostToDevice, s));
    if (nl) HK_TRY(cudaMemcpyAsync(lights, lights8, (size_t)nl * 32, cudaMemcpyHostToDevice, s));

    TraceLaunch L;
    memset(&L, 0, sizeof(L));
    L.nodes = reinterpret_cast<const uint2 *>(d_nodes2);
    L.refs = d_refs;
    L.tris = reinterpret_cast<const TriRec *>(d_records16);
    L.ntris = ntris;
    L.box = box;
    L.fetch = control;
    L.err = control + 1;
    L.counters = reinterpret_cast<unsigned long long *>(control + 4);
    L.stack_depth = 6;
    L.max_steps = 1u << 26;
    L.variant = (int)variant;
    L.count = false;
    L.block = 128;
    L.grid = sm * 16;
    HK_TRY(launch_camera_rays(cam, w, h, rays, s));
    L.rays = rays;
    L.hits = hits;
    L.n = (uint32_t)npix;
    L.n_dev = nullptr;
    HK_TRY(launch_trace(L, s));
    HK_TRY(launch_shadow_rays(rays, hits, L.tris, (uint32_t)npix, lights, nl, nullptr, srays, slot, spix, control + 2,
                              s));
    L.rays = srays;
    L.hits = shits;
    L.n = 0;
    L.n_dev = control + 2;
    L.occlusion = true;
    HK_TRY(launch_trace(L, s));
    HK_TRY(launch_shade_cpu(rays, hits, L.tris, (uint32_t)npix, lights, nl, slot, shits, d_rgba, s));
    uint32_t err = 0;
    HK_TRY(cudaMemcpyAsync(&err, control + 1, 4, cudaMemcpyDeviceToHost, s));
    HK_TRY(cudaStreamSynchronize(s));
#undef HK_TRY
    return err ? HK_E_BOUNDS : HK_OK;
}
