// noalloc.cu -- gpair_vis2data_chi2_noalloc: V2 / T3 mock data and chi2 from
// visibilities, for callers that cannot allocate device memory.
//
// Who cannot allocate. Some host programs hand the whole device heap to their
// own allocator up front: a framework's caching allocator, or a pipeline
// that reserves memory for many reconstructions at once. A cudaMalloc inside
// a library call then competes with that allocator. It can fail, or fragment
// the reserved pool. Other callers run this step inside a latency-critical
// loop, where cudaMalloc/cudaFree can serialise the device and stall work on
// other streams. This entry point therefore allocates nothing. The caller
// passes device buffers for every input and output. The kernel's only scratch
// (per-block FP64 partial sums of chi2 and an arrival counter) is a fixed
// file-scope device array that each GPU loading this library holds until the
// process exits.
//
// Same arithmetic as the data stage of the main path (k_vis_data): V2 for the
// first npow uv points, T3 = V~ab V~bc V~ca * phasor per triangle, chi2 as an
// FP64 deterministic sum. Inputs use the reference's device layouts
// (gpair1/trunk/gpair.c:574-608): visibilities float2[nuv], data/data_err
// float[npow + 2*nbis], phasor float2[nbis], uvpnt long4[nbis], sign short4[nbis].
#include <mutex>

#include "gpair_internal.cuh"

#define NOALLOC_THREADS 256
#define NOALLOC_MAX_BLOCKS 8192  // scratch holds one partial per block
#define NOALLOC_MAX_ITEMS ((long long)NOALLOC_MAX_BLOCKS * NOALLOC_THREADS)  // npow + nbis <= 2,097,152

// [0, 256): arrival counter (uint32) and error word (uint32); [256, ...): double partials
static __device__ __align__(256) unsigned char g_noalloc_scratch[256 + NOALLOC_MAX_BLOCKS * sizeof(double)];

__global__ void __launch_bounds__(NOALLOC_THREADS) k_vis2data_chi2_noalloc(
    unsigned char *__restrict__ scratch, const float2 *__restrict__ visi, int nuv, int npow, int nbis,
    const float *__restrict__ data, const float *__restrict__ data_err, const float2 *__restrict__ phasor,
    const longlong4 *__restrict__ uvpnt, const short4 *__restrict__ sign, float *__restrict__ mock,
    double *__restrict__ chi2_out)
{
    unsigned int *counter = reinterpret_cast<unsigned int *>(scratch);
    unsigned int *errword = counter + 1;
    double *partials = reinterpret_cast<double *>(scratch + 256);
    __shared__ double red[32];
    __shared__ bool am_last;
    double chi = 0.0;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < npow) {
        float2 v = visi[i];
        double m2 = (double)v.x * v.x + (double)v.y * v.y;
        mock[i] = (float)m2;
        double r = (m2 - (double)data[i]) * (double)data_err[i];
        chi = r * r;
    } else if (i < (long long)npow + nbis) {
        int t = (int)(i - npow);
        longlong4 q = uvpnt[t];
        short4 sg = sign[t];
        if (q.x < 0 || q.x >= nuv || q.y < 0 || q.y >= nuv || q.z < 0 || q.z >= nuv) {
            atomicOr(errword, 1u);  // out-of-range triangle reference: skip the access, flag it
        } else {
            float2 a = visi[q.x], b = visi[q.y], c = visi[q.z];
            double ar = a.x, ai = sg.x < 0 ? -a.y : a.y;
            double br = b.x, bi = sg.y < 0 ? -b.y : b.y;
            double cr = c.x, ci = sg.z < 0 ? -c.y : c.y;
            double abr = ar * br - ai * bi, abi = ar * bi + ai * br;
            double tr = abr * cr - abi * ci, ti = abr * ci + abi * cr;
            float2 ph = phasor[t];
            double t3r = tr * ph.x - ti * ph.y, t3i = tr * ph.y + ti * ph.x;
            int r0 = npow + 2 * t;
            mock[r0] = (float)t3r;
            mock[r0 + 1] = (float)t3i;
            double e0 = (t3r - (double)data[r0]) * (double)data_err[r0];
            double e1 = (t3i - (double)data[r0 + 1]) * (double)data_err[r0 + 1];
            chi = e0 * e0 + e1 * e1;
        }
    }
    // block sum (fixed tree), then the last block sums the partials in block order
    for (int off = 16; off > 0; off >>= 1) chi += __shfl_down_sync(0xffffffffu, chi, off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = chi;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
        partials[blockIdx.x] = s;
        __threadfence();
        am_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return;
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) s += __ldcg(&partials[b]);
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    __syncthreads();
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += red[w];
        *chi2_out = (__ldcg(errword) != 0u) ? __longlong_as_double(0x7ff8000000000000LL) : tot;
        *counter = 0u;
    }
}

// Device address of the scratch array, looked up once per device with that
// device current (host code cannot use the symbol itself as a device pointer).
static std::mutex g_noalloc_mu;
static void *g_noalloc_addr[128];

static int noalloc_scratch_for_current_device(void **addr)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return GPAIR_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return GPAIR_ERR_CUDA;
        g_noalloc_addr[dev] = p;
    }
    *addr = g_noalloc_addr[dev];
    return GPAIR_OK;
}

extern "C" int gpair_vis2data_chi2_noalloc(const gpair_float2 *visi, int nuv, int npow, int nbis, const float *data,
                                           const float *data_err, const gpair_float2 *phasor,
                                           const gpair_long4 *uvpnt, const gpair_short4 *sign, float *mock,
                                           double *chi2, void *stream)
{
    if (nuv < 0 || npow < 0 || nbis < 0 || npow > nuv || !chi2) return GPAIR_ERR_INVALID;
    long long items = (long long)npow + nbis;
    if (items > NOALLOC_MAX_ITEMS) return GPAIR_ERR_INVALID;  // beyond the fixed scratch: refuse
    if (items > 0 && (!visi || !data || !data_err || !mock)) return GPAIR_ERR_INVALID;
    if (nbis > 0 && (!phasor || !uvpnt || !sign)) return GPAIR_ERR_INVALID;
    void *scratch = nullptr;
    int rc = noalloc_scratch_for_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (s) {
        // the scratch address belongs to the current device: the stream must too
        int cur = -1, sdev = -1;
        if (cudaGetDevice(&cur) != cudaSuccess || cudaStreamGetDevice(s, &sdev) != cudaSuccess) return GPAIR_ERR_CUDA;
        if (sdev != cur) return GPAIR_ERR_INVALID;
    }
    // the counter and the error word must start at zero; the partials are overwritten
    if (cudaMemsetAsync(scratch, 0, 2 * sizeof(unsigned int), s) != cudaSuccess) return GPAIR_ERR_CUDA;
    int blocks = items > 0 ? (int)((items + NOALLOC_THREADS - 1) / NOALLOC_THREADS) : 1;
    k_vis2data_chi2_noalloc<<<blocks, NOALLOC_THREADS, 0, s>>>(
        (unsigned char *)scratch, (const float2 *)visi, nuv, npow, nbis, data, data_err, (const float2 *)phasor,
        (const longlong4 *)uvpnt, (const short4 *)sign, mock, chi2);
    return cudaGetLastError() == cudaSuccess ? GPAIR_OK : GPAIR_ERR_CUDA;
}
