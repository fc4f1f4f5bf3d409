// umma_dft.cu -- forward DFT and adjoint contraction on the 5th-generation
// tensor cores (tcgen05, TMEM accumulators, TMA operand staging).
//
// Precision (GPAIR_PREC_SPLIT16): every operand x is stored as a pair of f16
// values hi = f16(x), lo = f16(x - hi) after a power-of-two scaling that puts
// the operand near the top of the f16 range (twiddles: 2^10; the forward's
// image operand: one scale per image row, from the row's max; the adjoint's
// weights: one scale from max |c_k|); a product is formed as
// A_hi B_hi + A_hi B_lo + A_lo B_hi with FP32 accumulation (the lo*lo term is
// below 2^-22 of the result). Scales are exact powers of two and are removed
// in the epilogues. GPAIR_PREC_SPLIT16F8: the forward forms the two cross
// terms as E4M3 products (kind::f8f6f4) into the same accumulator (OP_F16F8).
//
// Both contractions put the twiddle-side table in the M operand (TMEM lanes:
// 128 rows on one CTA, 256 on a CTA pair) and the image-side operand in the
// N = 256 operand (TMEM columns).
// Forward DFT (kernel_visi.cl / cpu.c:449-475):
//   T[n][y] = sum_x Fx16[n][x] I[y][x],  row n = 2k+c holds (Re, Im) Fx[k][x]
//   epilogue: the thread of row n sums over its 128 columns against Fy (an
//   anchor every 16 rows, rotated within the chunk); the Re/Im row pair is
//   combined with one shuffle: Vpart[entry][k] = sum_y (T[2k][y] + i T[2k+1][y]) Fy[k][y],
//   one entry per 128 image rows (per image of a stack of smaller images)
// Adjoint (kernel_grad_pow.cl + kernel_grad_bis.cl / cpu.c:279-369):
//   G[y][x] = sum_k' FxT[x][k'] W[y][k'],  W[y][2k] = Re(c_k Fy[k][y]),
//   W[y][2k+1] = -Im(c_k Fy[k][y]),  FxT[x][2k+c] = (Re, Im) Fx[k][x]
//   the thread of image column x stores G[y][x] for its 128 rows (consecutive
//   lanes write consecutive x); split over k' into S partial images that
//   k_grad_finalize sums in a fixed order
//
// One persistent CTA per SM (or CTA pair per two SMs), 320 threads: warp 0
// issues TMA loads (a ring of 2 stages of 96 KB, or 3 of 64 KB per CTA of a
// pair), warp 1 owns TMEM (512 columns = two FP32 accumulators of 256
// columns) and one of its threads issues tcgen05.mma; warps 2-9 drain TMEM,
// two per lane quarter, each taking 128 of the accumulator's 256 columns.
// All waits are bounded; a timeout sets an error code, the roles stop, TMEM is
// released, and the host reports GPAIR_ERR_TIMEOUT.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cudaTypedefs.h>
#include <stdlib.h>
#include <string.h>

#include "gpair_internal.cuh"
#include "group.cuh"
#include "reduce.cuh"
#include "umma.cuh"

#define TC_BM 128
#define TC_BN 256
#define TC_ROWB 128  // bytes of one K-block row: 64 f16 or 32 TF32 elements
#define TC_STAGES 2
// warps: 0 TMA producer, 1 MMA issuer, then the epilogue warps: the forward has
// TC_EPI_WARPS, two per TMEM lane quarter, each with TC_EPI_COLS accumulator
// columns; the adjoint's store epilogue TC_STORE_WARPS, one per quarter (eight
// measured 35 % slower there: the extra warps share the issue slots of the TMA
// and MMA warps' sub-partitions while the units are MMA-bound)
#define TC_EPI_WARPS 8
#define TC_EPI_COLS (TC_BN * 4 / TC_EPI_WARPS)
#define TC_STORE_WARPS 4
#define TC_TW_LOG2 10  // twiddle operands are scaled by 2^10
#define TC_A_BYTES (TC_BM * TC_ROWB)
#define TC_B_BYTES (TC_BN * TC_ROWB)
#define TC_STAGE_BYTES (2 * TC_A_BYTES + 2 * TC_B_BYTES)
#define TC_TMEM_COLS 512
// after the stages: barriers (256 B), the unit prefix sums of a grouped launch
// (up to TC_GROUP_MAX instances), then the forward epilogue's row scales of a
// unit, one copy per epilogue warp and accumulator buffer
#define TC_RS_OFF (256 + 4 * 272)
#define TC_RS_BYTES (TC_EPI_WARPS * 2 * TC_EPI_COLS * 4)
#define TC_SMEM_BYTES (1024 + TC_STAGES * TC_STAGE_BYTES + TC_RS_OFF + TC_RS_BYTES)
#define TC_SMEM_GROUP_BYTES TC_SMEM_BYTES
#define TC_WAIT_BUDGET 4000000000LL  // default clock cycles (~2 s) per pipeline wait
#define RPMAS_TC ((3.14159265358979323 / 180.0) / 3600000.0)  // radians per milliarcsecond

enum { EPI_FWD = 0, EPI_STORE = 1 };

template <int EPI> constexpr int tc_epi_warps() { return EPI == EPI_FWD ? TC_EPI_WARPS : TC_STORE_WARPS; }
template <int EPI> constexpr int tc_threads() { return 64 + 32 * tc_epi_warps<EPI>(); }

// Operand element types: f16 (kind::f16, K = 16 per MMA) or TF32 held as FP32
// bit patterns (kind::tf32, K = 8 per MMA). Both fill 128-byte K-block rows,
// so the shared-memory stages, descriptors and TMA boxes are the same in bytes.
// OP_F16F8 (forward only): f16 hi operands for hi*hi (kind::f16) and 8-bit
// E4M3 operands for the two cross terms (kind::f8f6f4, K = 32 per MMA, twice
// the f16 rate), 64-byte rows with 64-byte swizzling; a K-block is 64 elements
// of each.
enum { OP_F16 = 0, OP_TF32 = 1, OP_F16F8 = 2 };
__host__ __device__ constexpr int tc_bk(int op) { return op == OP_TF32 ? 32 : 64; }

// E4M3 (round to nearest even, saturating at 448) of x
__device__ __forceinline__ uint8_t to_e4m3(float x)
{
    return (uint8_t)__nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
}
// Power-of-two scales of the 8-bit cross-term operands (E4M3 holds |x| <= 448
// with 3 mantissa bits): twiddle hi / 4 (|hi| <= 2^10), twiddle lo * 2^10
// (|lo| <= 2^-2), image hi / 2^10 (|hi| <= 2^15), image lo * 4 (|lo| <= 2^3).
// (A_hi / 4)(4 B_lo) = A_hi B_lo and (2^10 A_lo)(B_hi / 2^10) = A_lo B_hi, so the
// cross terms accumulate in the same FP32 accumulator as A_hi B_hi.
#define F8_A_HI 0.25f
#define F8_A_LO 1024.f
#define F8_B_HI (1.f / 1024.f)
#define F8_B_LO 4.f

// f16 hi of v and the 8-bit pair (hi * s_hi, (v - hi) * s_lo)
__device__ __forceinline__ void split_f8(float v, float s_hi, float s_lo, __half &h, uint8_t &q_hi, uint8_t &q_lo)
{
    h = __float2half_rn(v);
    const float hf = __half2float(h);
    q_hi = to_e4m3(hf * s_hi);
    q_lo = to_e4m3((v - hf) * s_lo);
}
// products per K step: 3 = hi*hi + hi*lo + lo*hi of split operands, 1 = hi*hi
// At most TC_SPLIT_PRODUCTS products per adjoint split-K partial (FP32 accumulation)
#define TC_SPLIT_PRODUCTS 4096

template <typename OT> struct OpSplit;
template <> struct OpSplit<__half> {
    // f16 hi = f16(v), lo = f16(v - hi)
    static __device__ __forceinline__ void split(float v, __half &h, __half &l)
    {
        h = __float2half_rn(v);
        l = __float2half_rn(v - __half2float(h));
    }
};
template <> struct OpSplit<float> {
    // TF32 hi = tf32(v), lo = tf32(v - hi) (v - hi is exact in FP32)
    static __device__ __forceinline__ void split(float v, float &h, float &l)
    {
        h = umma::tf32_rna(v);
        l = umma::tf32_rna(v - h);
    }
};

template <typename OT>
__device__ __forceinline__ void split_store(OT *__restrict__ hi, OT *__restrict__ lo, size_t i, float v)
{
    OT h, l;
    OpSplit<OT>::split(v, h, l);
    hi[i] = h;
    if (lo) lo[i] = l;
}

struct TcArgs {
    int m_tiles, n_tiles, kb_total, kb_per_split, units;
    // forward epilogue: Fy[k][16 j] anchors, per-uv rotation e^{-2 pi i s v_k}
    const float2 *fya, *fyr;
    int nanc;
    int N, nuv;
    // image-side rows: lpad rows per image, partial entries of 2^elog2 rows;
    // rsc[row]: power-of-two factor of every image-side row (operand scale and
    // twiddle scale removed in the epilogue)
    int lpad, elog2;
    const float *rsc;
    float2 *vpart;
    // store epilogue
    float *gpart;
    int out_ld, out_rows, out_cols;
    unsigned int *err;
    // clock budget of each pipeline wait; the drain of the TMA copies in
    // flight always keeps TC_WAIT_BUDGET, so that no copy is outstanding when
    // the CTA retires. skip_loads: the producer issues no TMA loads (used to
    // make the other roles' waits run out with nothing in flight)
    long long budget;
    int skip_loads;
    // grouped forward (GROUP = 1): ninst instances, the units of instance i
    // taken when gate[i] != 0
    const struct TcGroupInst *grp;
    const int *gate;
    int ninst;
};

// One instance of a grouped forward launch: its operand maps (the twiddles and
// the stacked trial images of its batched line search) and its epilogue
// arguments. Held in global memory; the maps are read through their generic
// addresses.
struct __align__(64) TcGroupInst {
    CUtensorMap A_hi, A_lo, A_x, B_hi, B_lo, B_x;  // A_x, B_x: OP_F16F8's second 8-bit operands
    int m_tiles, n_tiles, kb_total, units;
    // forward epilogue
    const float2 *fya, *fyr;
    int nanc, nuv, lpad, elog2;
    const float *rsc;
    float2 *vpart;
    // store epilogue (adjoint): split-K partial images
    int kb_per_split;
    float *gpart;
    int out_ld, out_rows, out_cols;
};
#define TC_GROUP_MAX 256  // instances of one grouped launch (prefix sums in shared memory)

struct TcState {
    // A side (M = 128 rows): forward twiddles [rows_pad][Kx_pad], adjoint twiddles [xrows_pad][K2_pad]
    // B side (N = 256 rows): image [M_pad][Kx_pad], adjoint weights [M_pad][K2_pad]
    // batched trials: GP_NTR images stacked at Lb rows each, [GP_NTR Lb][Kx_pad]
    // op: OP_F16 or OP_TF32 (element size esz, bk elements per K-block);
    // nprod: 3 (split operands; the lo buffers exist) or 1 (hi only);
    // fop: the forward's operand kind (op, or OP_F16F8: the forward's lo
    // operands are the E4M3 buffers *8h / *8l, its f16 lo buffers do not exist)
    int op, nprod, esz, bk, fop;
    void *fx8h, *fx8l, *img8h, *img8l, *imgb8h, *imgb8l;
    CUtensorMap m_fx8h, m_fx8l, m_img8h, m_img8l, m_imgb8h, m_imgb8l;
    int Kx_pad, M_pad, rows_pad, K2_pad, xrows_pad;
    int Lb, epp_b;
    void *imgb_hi, *imgb_lo;
    CUtensorMap m_imgb_hi, m_imgb_lo;
    // power-of-two factor of every image-side operand row: single image
    // [M_pad], batch stack [GP_NTR Lb] (zero on padding rows)
    float *rsc, *rscb;
    int splits, kb_per;
    void *img_hi, *img_lo, *fx_hi, *fx_lo, *fxt_hi, *fxt_lo, *w_hi, *w_lo;
    float2 *fya, *fyr;
    int nanc;
    CUtensorMap m_img_hi, m_img_lo, m_fx_hi, m_fx_lo, m_w_hi, m_w_lo, m_fxt_hi, m_fxt_lo;
    int nsm;
    // CTA pairs (cta_group::2): B maps with 128-row boxes, A row counts padded
    // to 256; npairs = clusters of two that are resident at once
    int pair, npairs;
};

static inline int round_up(long long a, long long b) { return (int)(((a + b - 1) / b) * b); }

// ------------------------------------------------------------------ GEMM

__device__ __forceinline__ void tc_fail(unsigned int *err, volatile int *abort_flag, unsigned int code)
{
    atomicOr(err, code);
    *abort_flag = 1;
}

// One step of Fy along y: w * e^{-2 pi i s v_k}, with the rounding fixed (one
// rounded product, then one fused multiply-add per component)
__device__ __forceinline__ float2 fy_step(float2 w, float2 rot)
{
    return make_float2(fmaf(w.x, rot.x, -__fmul_rn(w.y, rot.y)), fmaf(w.x, rot.y, __fmul_rn(w.y, rot.x)));
}

template <int EPI>
__device__ __forceinline__ void tc_decode(const TcArgs &a, int u, int &m, int &n, int &kb0, int &kb1, int &split)
{
    n = u % a.n_tiles;
    int rest = u / a.n_tiles;
    if (EPI == EPI_FWD) {
        m = rest;
        split = 0;
        kb0 = 0;
        kb1 = a.kb_total;
    } else {
        m = rest % a.m_tiles;
        split = rest / a.m_tiles;
        kb0 = split * a.kb_per_split;
        kb1 = min(a.kb_total, kb0 + a.kb_per_split);
    }
}

// Unit u of a launch: tile (m, n), K-blocks [kb0, kb1), split. GROUP = 1: u
// counts the units of the gated instances in instance order (prefix sums
// gpre[0..ninst]); `ci` is the caller's instance cursor, which only moves
// forward because every role visits its units in increasing order.
template <int EPI, int GROUP>
__device__ __forceinline__ void tc_unit(const TcArgs &a, const int *gpre, int u, int &ci, int &m, int &n, int &kb0,
                                        int &kb1, int &split)
{
    if (GROUP) {
        while (gpre[ci + 1] <= u) ci++;
        const TcGroupInst &gi = a.grp[ci];
        const int lu = u - gpre[ci], nt = gi.n_tiles;
        n = lu % nt;
        if (EPI == EPI_FWD) {
            m = lu / nt;
            split = 0;
            kb0 = 0;
            kb1 = gi.kb_total;
        } else {
            const int rest = lu / nt;
            m = rest % gi.m_tiles;
            split = rest / gi.m_tiles;
            kb0 = split * gi.kb_per_split;
            kb1 = min(gi.kb_total, kb0 + gi.kb_per_split);
        }
    } else {
        tc_decode<EPI>(a, u, m, n, kb0, kb1, split);
    }
}

// PAIR = 0: one CTA per tile of 128 (A rows) x 256 (B rows), 2 stages of 96 KB.
// PAIR = 1: a cluster of two CTAs shares one tcgen05.mma.cta_group::2 tile of
// 256 x 256: each CTA stages 128 rows of A and 128 rows of B (half of the tile's
// B) per K-block in its own shared memory, 3 stages of 64 KB, and holds 128
// TMEM lanes of the accumulator. The even CTA issues the MMAs; the odd CTA's
// TMA loads report to the even CTA's full barriers, the MMA commits release
// the stages of both CTAs, and both CTAs' epilogues release the even CTA's
// accumulator buffers. Per SM the operand traffic per MMA drops by a third.
template <int PAIR> struct TcGeo {
    static constexpr int MT = PAIR ? 256 : 128;          // M rows per tile (per unit)
    static constexpr int BROWS = PAIR ? 128 : 256;       // B rows staged per CTA
    static constexpr int B_BYTES = BROWS * TC_ROWB;
    static constexpr int STAGE = 2 * TC_A_BYTES + 2 * B_BYTES;
    static constexpr int STAGES = PAIR ? 3 : 2;
};
static_assert(TcGeo<0>::STAGES * TcGeo<0>::STAGE == TcGeo<1>::STAGES * TcGeo<1>::STAGE, "same smem in both modes");

// GROUP = 1: one launch over the units of several instances (TcGroupInst),
// each with its own maps and epilogue arguments; the kernel's map parameters
// are not used.
//
// OP_F16F8: each stage holds A_hi (f16, 128-byte rows), A8_hi and A8_lo (E4M3,
// 64-byte rows), B_hi, B8_hi and B8_lo; per K-block 4 kind::f16 MMAs (A_hi B_hi)
// and 2 x 2 kind::f8f6f4 MMAs (A8_hi B8_lo, A8_lo B8_hi), same stage bytes as
// the three f16 products. Maps: (A_hi, A_lo, A_x) = (f16 hi, E4M3 hi, E4M3 lo)
// and likewise for B; A_x and B_x are not used by the other operand kinds.
template <int EPI, int OP, int NPROD, int PAIR, int GROUP>
__global__ void __launch_bounds__(tc_threads<EPI>(), 1)
    k_tc_gemm(const __grid_constant__ CUtensorMap tA_hi, const __grid_constant__ CUtensorMap tA_lo,
              const __grid_constant__ CUtensorMap tA_x, const __grid_constant__ CUtensorMap tB_hi,
              const __grid_constant__ CUtensorMap tB_lo, const __grid_constant__ CUtensorMap tB_x, const TcArgs a)
{
    static_assert(OP != OP_F16F8 || (EPI == EPI_FWD && NPROD == 3), "the 8-bit cross terms serve the forward");
    constexpr bool F8 = OP == OP_F16F8;
    gp_pdl_enter();  // operands and gates come from the kernels before it
    using G = TcGeo<PAIR>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *stages = smem;
    uint64_t *full = (uint64_t *)(smem + G::STAGES * G::STAGE);
    uint64_t *empty = full + G::STAGES;
    uint64_t *tfull = empty + G::STAGES;
    uint64_t *tempty = tfull + 2;
    uint64_t *done_bar = tempty + 2;
    uint32_t *tmem_slot = (uint32_t *)(done_bar + 1);
    volatile int *abort_flag = (volatile int *)(tmem_slot + 1);
    int *gpre = (int *)(smem + G::STAGES * G::STAGE + 256);  // GROUP: unit prefix sums
    float *rsbuf = (float *)(smem + G::STAGES * G::STAGE + TC_RS_OFF);  // forward: row scales of a unit

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = PAIR ? umma::cluster_ctarank() : 0u;
    const bool leader = rank == 0;
    const int unit0 = PAIR ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;  // this CTA's (pair's) first unit
    const int ustep = PAIR ? (int)(gridDim.x >> 1) : (int)gridDim.x;
    if (threadIdx.x == 0) {
        for (int s = 0; s < G::STAGES; s++) {
            umma::mbar_init(&full[s], 1);
            umma::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            umma::mbar_init(&tfull[b], 1);
            umma::mbar_init(&tempty[b], (PAIR ? 2 : 1) * 32 * tc_epi_warps<EPI>());  // pair: both CTAs' epilogues release
        }
        umma::mbar_init(done_bar, 1);
        *abort_flag = 0;
        umma::fence_barrier_init();
    }
    if (GROUP) {
        // units of the gated instances, then their prefix sums (warp 0, 32 at a time)
        for (int i = threadIdx.x; i < a.ninst; i += blockDim.x) gpre[i + 1] = a.gate[i] ? a.grp[i].units : 0;
        __syncthreads();
        if (warp == 0) {
            int carry = 0;
            for (int b = 0; b < a.ninst; b += 32) {
                int v = b + lane < a.ninst ? gpre[b + lane + 1] : 0;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const int o = __shfl_up_sync(0xffffffffu, v, off);
                    if (lane >= off) v += o;
                }
                if (b + lane < a.ninst) gpre[b + lane + 1] = v + carry;
                carry += __shfl_sync(0xffffffffu, v, 31);
            }
            if (lane == 0) gpre[0] = 0;
        }
    }
    if (warp == 1) {
        if (PAIR) {
            umma::tmem_alloc_pair(tmem_slot, TC_TMEM_COLS);
            umma::tmem_relinquish_pair();
        } else {
            umma::tmem_alloc(tmem_slot, TC_TMEM_COLS);
            umma::tmem_relinquish();
        }
    }
    umma::tc_fence_before();
    __syncthreads();
    if (PAIR) umma::cluster_sync_all();  // both CTAs' barriers initialised before any remote arrival
    umma::tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int units = GROUP ? gpre[a.ninst] : a.units;

    if (warp == 0) {
        if (lane == 0) {
            // ------------------------------------------------ TMA producer
            const CUtensorMap *mAh = &tA_hi, *mAl = &tA_lo, *mAx = &tA_x, *mBh = &tB_hi, *mBl = &tB_lo, *mBx = &tB_x;
            if (!GROUP) {
                umma::tma_prefetch(mAh);
                umma::tma_prefetch(mAl);
                umma::tma_prefetch(mBh);
                umma::tma_prefetch(mBl);
                if (F8) {
                    umma::tma_prefetch(mAx);
                    umma::tma_prefetch(mBx);
                }
            }
            const uint32_t tx = (NPROD == 3 ? G::STAGE : TC_A_BYTES + G::B_BYTES) * (PAIR ? 2 : 1);
            int it = 0, ci = 0, cur = -1;
            for (int u = unit0; u < units && !*abort_flag; u += ustep) {
                int m, n, kb0, kb1, split;
                tc_unit<EPI, GROUP>(a, gpre, u, ci, m, n, kb0, kb1, split);
                if (GROUP && ci != cur) {
                    // this instance's maps, written to global memory before the launch
                    cur = ci;
                    mAh = &a.grp[ci].A_hi;
                    mAl = &a.grp[ci].A_lo;
                    mAx = &a.grp[ci].A_x;
                    mBh = &a.grp[ci].B_hi;
                    mBl = &a.grp[ci].B_lo;
                    mBx = &a.grp[ci].B_x;
                    umma::tensormap_acquire(mAh);
                    umma::tensormap_acquire(mAl);
                    umma::tensormap_acquire(mBh);
                    umma::tensormap_acquire(mBl);
                    if (F8) {
                        umma::tensormap_acquire(mAx);
                        umma::tensormap_acquire(mBx);
                    }
                }
                const int arow0 = m * G::MT + (int)rank * 128, brow0 = n * TC_BN + (int)rank * G::BROWS;
                for (int kb = kb0; kb < kb1; kb++) {
                    const int s = it % G::STAGES;
                    const uint32_t ph = (uint32_t)(it / G::STAGES) & 1u;
                    if (!umma::mbar_wait(&empty[s], ph ^ 1u, a.budget)) {
                        tc_fail(a.err, abort_flag, 1u);
                        break;
                    }
                    if (a.skip_loads) continue;  // nothing issued: the stage never fills
                    unsigned char *st = stages + s * G::STAGE;
                    const int kx = kb * tc_bk(OP);
                    if (PAIR) {
                        // both CTAs' bytes are counted on the leader's barrier
                        const uint32_t fb = umma::mapa_shared(umma::smem_u32(&full[s]), 0);
                        if (leader) umma::mbar_arrive_expect_tx(&full[s], tx);
                        umma::tma_load_2d_pair(st, mAh, fb, kx, arow0);
                        umma::tma_load_2d_pair(st + 2 * TC_A_BYTES, mBh, fb, kx, brow0);
                        if (F8) {
                            // the 8-bit tiles: 64-byte rows, half the bytes of an f16 tile
                            umma::tma_load_2d_pair(st + TC_A_BYTES, mAl, fb, kx, arow0);
                            umma::tma_load_2d_pair(st + TC_A_BYTES + TC_A_BYTES / 2, mAx, fb, kx, arow0);
                            umma::tma_load_2d_pair(st + 2 * TC_A_BYTES + G::B_BYTES, mBl, fb, kx, brow0);
                            umma::tma_load_2d_pair(st + 2 * TC_A_BYTES + G::B_BYTES + G::B_BYTES / 2, mBx, fb, kx,
                                                   brow0);
                        } else if (NPROD == 3) {
                            umma::tma_load_2d_pair(st + TC_A_BYTES, mAl, fb, kx, arow0);
                            umma::tma_load_2d_pair(st + 2 * TC_A_BYTES + G::B_BYTES, mBl, fb, kx, brow0);
                        }
                    } else {
                        umma::mbar_arrive_expect_tx(&full[s], tx);
                        umma::tma_load_2d(st, mAh, &full[s], kx, arow0);
                        umma::tma_load_2d(st + 2 * TC_A_BYTES, mBh, &full[s], kx, brow0);
                        if (F8) {
                            umma::tma_load_2d(st + TC_A_BYTES, mAl, &full[s], kx, arow0);
                            umma::tma_load_2d(st + TC_A_BYTES + TC_A_BYTES / 2, mAx, &full[s], kx, arow0);
                            umma::tma_load_2d(st + 2 * TC_A_BYTES + G::B_BYTES, mBl, &full[s], kx, brow0);
                            umma::tma_load_2d(st + 2 * TC_A_BYTES + G::B_BYTES + G::B_BYTES / 2, mBx, &full[s], kx,
                                              brow0);
                        } else if (NPROD == 3) {
                            umma::tma_load_2d(st + TC_A_BYTES, mAl, &full[s], kx, arow0);
                            umma::tma_load_2d(st + 2 * TC_A_BYTES + G::B_BYTES, mBl, &full[s], kx, brow0);
                        }
                    }
                    it++;
                }
            }
            // no copy may be in flight when the CTA retires: wait for the last
            // load issued into each stage (bounded; `it` counts issued stages).
            // With a pair the leader's barriers count both CTAs' copies, and the
            // odd CTA retires only after the cluster barrier below.
            if (leader)
                for (int j = 1; j <= G::STAGES && it - j >= 0; j++) {
                    const int i = it - j, s = i % G::STAGES;
                    if (!umma::mbar_wait(&full[s], (uint32_t)(i / G::STAGES) & 1u, TC_WAIT_BUDGET))
                        tc_fail(a.err, abort_flag, 16u);
                }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0 && leader) {
            // ------------------------------------------------ MMA issuer
            const uint32_t idesc = umma::idesc_f16(G::MT, TC_BN, OP == OP_TF32 ? 2 : 0);  // f16, tf32; E4M3 for f8f6f4
            int it = 0, t = 0, ci = 0;
            bool ok = true, issued = false;
            for (int u = unit0; u < units && ok && !*abort_flag; u += ustep, t++) {
                int m, n, kb0, kb1, split;
                tc_unit<EPI, GROUP>(a, gpre, u, ci, m, n, kb0, kb1, split);
                const int b = t & 1;
                if (!umma::mbar_wait(&tempty[b], ((uint32_t)(t >> 1) & 1u) ^ 1u, a.budget)) {
                    tc_fail(a.err, abort_flag, 2u);
                    break;
                }
                umma::tc_fence_after();
                const uint32_t d = tmem_base + (uint32_t)(b * TC_BN);
                for (int kb = kb0; kb < kb1; kb++, it++) {
                    const int s = it % G::STAGES;
                    if (!umma::mbar_wait(&full[s], (uint32_t)(it / G::STAGES) & 1u, a.budget)) {
                        tc_fail(a.err, abort_flag, 4u);
                        ok = false;
                        break;
                    }
                    umma::tc_fence_after();
                    unsigned char *st = stages + s * G::STAGE;
                    const uint64_t dah = umma::smem_desc_k_sw128(st);
                    const uint64_t dal = umma::smem_desc_k_sw128(st + TC_A_BYTES);
                    const uint64_t dbh = umma::smem_desc_k_sw128(st + 2 * TC_A_BYTES);
                    const uint64_t dbl = umma::smem_desc_k_sw128(st + 2 * TC_A_BYTES + G::B_BYTES);
                    if (F8) {
                        // hi*hi in f16, then the cross terms A8_hi B8_lo + A8_lo B8_hi in E4M3
                        const uint64_t qah = umma::smem_desc_k_sw64(st + TC_A_BYTES);
                        const uint64_t qal = umma::smem_desc_k_sw64(st + TC_A_BYTES + TC_A_BYTES / 2);
                        const uint64_t qbh = umma::smem_desc_k_sw64(st + 2 * TC_A_BYTES + G::B_BYTES);
                        const uint64_t qbl = umma::smem_desc_k_sw64(st + 2 * TC_A_BYTES + G::B_BYTES + G::B_BYTES / 2);
#pragma unroll
                        for (int kk = 0; kk < TC_ROWB / 32; kk++) {
                            const uint64_t off = (uint64_t)(kk * 32) >> 4;
                            const uint32_t acc = (kb > kb0 || kk > 0) ? 1u : 0u;
                            if (PAIR) umma::mma_f16_pair(d, dah + off, dbh + off, idesc, acc);
                            else umma::mma_f16_ss(d, dah + off, dbh + off, idesc, acc);
                        }
#pragma unroll
                        for (int kk = 0; kk < 2; kk++) {  // 32 E4M3 elements (32 B) per MMA
                            const uint64_t off = (uint64_t)(kk * 32) >> 4;
                            if (PAIR) {
                                umma::mma_f8_pair(d, qah + off, qbl + off, idesc, 1u);
                                umma::mma_f8_pair(d, qal + off, qbh + off, idesc, 1u);
                            } else {
                                umma::mma_f8_ss(d, qah + off, qbl + off, idesc, 1u);
                                umma::mma_f8_ss(d, qal + off, qbh + off, idesc, 1u);
                            }
                        }
                    } else {
#pragma unroll
                        for (int kk = 0; kk < TC_ROWB / 32; kk++) {
                            // one MMA covers 32 B along K: 16 f16 or 8 TF32 elements
                            const uint64_t off = (uint64_t)(kk * 32) >> 4;
                            const uint32_t acc = (kb > kb0 || kk > 0) ? 1u : 0u;
                            if (PAIR) {
                                if (OP == OP_F16) {
                                    umma::mma_f16_pair(d, dah + off, dbh + off, idesc, acc);
                                    if (NPROD == 3) {
                                        umma::mma_f16_pair(d, dah + off, dbl + off, idesc, 1u);
                                        umma::mma_f16_pair(d, dal + off, dbh + off, idesc, 1u);
                                    }
                                } else {
                                    umma::mma_tf32_pair(d, dah + off, dbh + off, idesc, acc);
                                    if (NPROD == 3) {
                                        umma::mma_tf32_pair(d, dah + off, dbl + off, idesc, 1u);
                                        umma::mma_tf32_pair(d, dal + off, dbh + off, idesc, 1u);
                                    }
                                }
                            } else if (OP == OP_F16) {
                                umma::mma_f16_ss(d, dah + off, dbh + off, idesc, acc);
                                if (NPROD == 3) {
                                    umma::mma_f16_ss(d, dah + off, dbl + off, idesc, 1u);
                                    umma::mma_f16_ss(d, dal + off, dbh + off, idesc, 1u);
                                }
                            } else {
                                umma::mma_tf32_ss(d, dah + off, dbh + off, idesc, acc);
                                if (NPROD == 3) {
                                    umma::mma_tf32_ss(d, dah + off, dbl + off, idesc, 1u);
                                    umma::mma_tf32_ss(d, dal + off, dbh + off, idesc, 1u);
                                }
                            }
                        }
                    }
                    issued = true;
                    // stage reusable (in both CTAs of a pair) once these MMAs finish
                    if (PAIR) umma::mma_commit_pair(&empty[s], 0x3);
                    else umma::mma_commit(&empty[s]);
                }
                if (!ok) break;
                // accumulator ready for the epilogue(s)
                if (PAIR) umma::mma_commit_pair(&tfull[b], 0x3);
                else umma::mma_commit(&tfull[b]);
            }
            // every MMA has completed before TMEM is released (a grouped launch can
            // leave a CTA without units: then nothing was issued)
            if (issued) {
                if (PAIR) umma::mma_commit_pair(done_bar, 0x1);
                else umma::mma_commit(done_bar);
                if (!umma::mbar_wait(done_bar, 0u, TC_WAIT_BUDGET)) tc_fail(a.err, abort_flag, 32u);
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------- epilogue
        const int ew = warp - 2;                 // epilogue warp
        const int q = warp & 3;                  // TMEM lane quarter this warp may access
        constexpr int ECOLS = TC_BN * 4 / tc_epi_warps<EPI>();  // accumulator columns per epilogue warp
        const int c0 = (ew >> 2) * ECOLS;                        // its first accumulator column
        // the accumulator buffers are released on the leader's barriers
        const uint32_t te0 = PAIR ? umma::mapa_shared(umma::smem_u32(&tempty[0]), 0) : 0u;
        const uint32_t te1 = PAIR ? umma::mapa_shared(umma::smem_u32(&tempty[1]), 0) : 0u;
        int t = 0, ci = 0;
        for (int u = unit0; u < units; u += ustep, t++) {
            int m, n, kb0, kb1, split;
            tc_unit<EPI, GROUP>(a, gpre, u, ci, m, n, kb0, kb1, split);
            const int b = t & 1;
            const int arow = m * G::MT + (int)rank * 128 + q * 32 + lane;  // row of the twiddle-side operand
            const int y0 = n * TC_BN;                                      // first image row of the columns
            const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * TC_BN + c0);
            if (EPI == EPI_FWD) {
                // Fy[k][y] along this thread's TC_EPI_COLS columns: an FP64-accurate anchor
                // every 16 rows, rotated by r_k = e^{-2 pi i s v_k} within the chunk (<= 15
                // steps). Partial entries hold at most TC_EPI_COLS rows (elog2 <= 7), so
                // that no entry spans two epilogue warps.
                const float2 *fya = a.fya, *fyr = a.fyr;
                const float *rsc = a.rsc;
                float2 *vpart = a.vpart;
                int nuv = a.nuv, nanc = a.nanc, lpad = a.lpad, elog2 = a.elog2;
                if (GROUP) {
                    const TcGroupInst &gi = a.grp[ci];
                    fya = gi.fya;
                    fyr = gi.fyr;
                    rsc = gi.rsc;
                    vpart = gi.vpart;
                    nuv = gi.nuv;
                    nanc = gi.nanc;
                    lpad = gi.lpad;
                    elog2 = gi.elog2;
                }
                const int k = arow >> 1;
                const bool vk = k < nuv;
                const float2 rot = vk ? __ldg(&fyr[k]) : make_float2(0.f, 0.f);
                const float2 *anc = fya + (size_t)(vk ? k : 0) * nanc;
                float2 an[TC_EPI_COLS / 16];
#pragma unroll
                for (int c = 0; c < TC_EPI_COLS / 16; c++) {
                    const int j = ((y0 + c0 + 16 * c) % lpad) >> 4;  // anchor of the row within its image
                    an[c] = (vk && j < nanc) ? __ldg(&anc[j]) : make_float2(0.f, 0.f);
                }
                // the row scales of this warp's columns into its shared copy (one L2
                // round trip per unit, issued before the accumulator is ready; the copy
                // of buffer b was last read by this warp two units ago)
                float *rsw = rsbuf + (ew * 2 + b) * TC_EPI_COLS;
                __syncwarp();
                {
                    static_assert(TC_EPI_COLS == 128, "one float4 per lane");
                    const float4 *src = reinterpret_cast<const float4 *>(rsc + y0 + c0);
                    reinterpret_cast<float4 *>(rsw)[lane] = __ldg(src + lane);
                }
                __syncwarp();
                if (!umma::mbar_wait(&tfull[b], (uint32_t)(t >> 1) & 1u, a.budget)) {
                    tc_fail(a.err, abort_flag, 8u);
                    break;
                }
                umma::tc_fence_after();
                const int emask = (1 << elog2) - 1;
                if (lpad < TC_EPI_COLS) {
                    // several images in this warp's columns (a batch stack of lpad = 32 or
                    // 64 rows each; y0 + c0 is a multiple of lpad): chunk q of every image
                    // has the same 16 values of Fy, formed once for all of them. Each
                    // image's sum takes its chunks and rows in the order of the loop below.
                    const int per = lpad >> 4, nimg = TC_EPI_COLS / lpad;
                    float are[TC_EPI_COLS / 32], aim[TC_EPI_COLS / 32];
#pragma unroll
                    for (int i = 0; i < TC_EPI_COLS / 32; i++) {
                        are[i] = 0.f;
                        aim[i] = 0.f;
                    }
#pragma unroll 1
                    for (int qq = 0; qq < per; qq++) {  // a loop, not unrolled: the tile code stays in the instruction cache
                        float2 wv[16];
                        wv[0] = (vk && qq < nanc) ? __ldg(&anc[qq]) : make_float2(0.f, 0.f);
#pragma unroll
                        for (int j = 1; j < 16; j++) wv[j] = fy_step(wv[j - 1], rot);
#pragma unroll
                        for (int ti = 0; ti < TC_EPI_COLS / 32; ti++) {
                            if (ti < nimg) {  // warp-uniform
                                const int c = ti * per + qq;
                                uint32_t r[16];
                                umma::tmem_ld16(taddr + (uint32_t)(c * 16), r);
                                float rs[16];
                                const float4 *rp = reinterpret_cast<const float4 *>(rsw + 16 * c);
#pragma unroll
                                for (int v4 = 0; v4 < 4; v4++) *reinterpret_cast<float4 *>(&rs[4 * v4]) = rp[v4];
                                umma::tmem_ld_wait();
                                float sr = are[ti], si = aim[ti];
#pragma unroll
                                for (int j = 0; j < 16; j++) {
                                    const float tv = __uint_as_float(r[j]) * rs[j];
                                    sr = fmaf(tv, wv[j].x, sr);
                                    si = fmaf(tv, wv[j].y, si);
                                }
                                are[ti] = sr;
                                aim[ti] = si;
                            }
                        }
                    }
#pragma unroll
                    for (int ti = 0; ti < TC_EPI_COLS / 32; ti++) {
                        if (ti < nimg) {
                            const int entry = (y0 + c0 + ti * lpad) >> elog2;
                            const float re = are[ti], im = aim[ti];
                            const float ore = __shfl_xor_sync(0xffffffffu, re, 1);
                            const float oim = __shfl_xor_sync(0xffffffffu, im, 1);
                            if ((lane & 1) == 0 && vk)
                                vpart[(size_t)entry * nuv + k] = make_float2(re - oim, im + ore);
                        }
                    }
                } else {
                    float sre = 0.f, sim = 0.f;
#pragma unroll
                    for (int c = 0; c < TC_EPI_COLS / 16; c++) {
                        uint32_t r[16];
                        umma::tmem_ld16(taddr + (uint32_t)(c * 16), r);
                        // power-of-two scales of the 16 image rows (shared memory, same address in every lane)
                        float rs[16];
                        const float4 *rp = reinterpret_cast<const float4 *>(rsw + 16 * c);
#pragma unroll
                        for (int v4 = 0; v4 < 4; v4++) *reinterpret_cast<float4 *>(&rs[4 * v4]) = rp[v4];
                        umma::tmem_ld_wait();
                        float2 w = an[c];
#pragma unroll
                        for (int j = 0; j < 16; j++) {
                            const float tv = __uint_as_float(r[j]) * rs[j];
                            sre = fmaf(tv, w.x, sre);
                            sim = fmaf(tv, w.y, sim);
                            w = fy_step(w, rot);
                        }
                        if (((y0 + c0 + 16 * c + 16) & emask) == 0) {
                            // end of a partial entry (warp-uniform): combine the Re/Im row
                            // pair, store. even row: (sum T_re F_re, sum T_re F_im);
                            // odd row: (sum T_im F_re, sum T_im F_im)
                            const int entry = (y0 + c0 + 16 * c) >> elog2;
                            const float re = sre, im = sim;
                            const float ore = __shfl_xor_sync(0xffffffffu, re, 1);
                            const float oim = __shfl_xor_sync(0xffffffffu, im, 1);
                            if ((lane & 1) == 0 && vk) vpart[(size_t)entry * nuv + k] = make_float2(re - oim, im + ore);
                            sre = 0.f;
                            sim = 0.f;
                        }
                    }
                }
            } else {
                if (!umma::mbar_wait(&tfull[b], (uint32_t)(t >> 1) & 1u, a.budget)) {
                    tc_fail(a.err, abort_flag, 8u);
                    break;
                }
                umma::tc_fence_after();
                float *gpart = a.gpart;
                int out_ld = a.out_ld, out_rows = a.out_rows, out_cols = a.out_cols;
                if (GROUP) {
                    const TcGroupInst &gi = a.grp[ci];
                    gpart = gi.gpart;
                    out_ld = gi.out_ld;
                    out_rows = gi.out_rows;
                    out_cols = gi.out_cols;
                }
                float *out = gpart + (size_t)split * out_rows * out_ld;
                const int x = arow;
                const bool xv = x < out_cols;
#pragma unroll 1
                for (int c = 0; c < ECOLS / 16; c++) {
                    uint32_t r[16];
                    umma::tmem_ld16(taddr + (uint32_t)(c * 16), r);
                    umma::tmem_ld_wait();
                    if (xv) {
#pragma unroll
                        for (int j = 0; j < 16; j++) {
                            const int y = y0 + c0 + c * 16 + j;
                            if (y < out_rows) out[(size_t)y * out_ld + x] = __uint_as_float(r[j]);
                        }
                    }
                }
            }
            umma::tc_fence_before();
            if (PAIR) umma::mbar_arrive_cluster(b ? te1 : te0);
            else umma::mbar_arrive(&tempty[b]);
        }
    }
    __syncthreads();
    // a pair retires together: no CTA leaves while the other may still touch its
    // shared memory, barriers or tensor memory
    if (PAIR) umma::cluster_sync_all();
    if (warp == 1) {
        umma::tc_fence_after();
        if (PAIR) umma::tmem_dealloc_pair(tmem_base, TC_TMEM_COLS);
        else umma::tmem_dealloc(tmem_base, TC_TMEM_COLS);
    }
}

// ------------------------------------------------------ operand kernels

// Twiddle operands: forward B [rows_pad][Kx_pad] (row 2k+c = Re/Im of Fx[k][:])
// and adjoint B [xrows_pad][K2_pad] (row x, column 2k+c), both scaled by 2^10.
// lo == nullptr: hi only (one-product mode). fx8 != nullptr (OP_F16F8): the
// forward's E4M3 pair (hi / 4, lo * 2^10) instead of its f16 lo.
template <typename OT>
__global__ void k_tc_twiddle_ops(const float2 *__restrict__ fx, int nuv, int N, int Kx_pad, int rows_pad,
                                 int K2_pad, int xrows_pad, OT *__restrict__ fx_hi, OT *__restrict__ fx_lo,
                                 uint8_t *__restrict__ fx8h, uint8_t *__restrict__ fx8l, OT *__restrict__ fxt_hi,
                                 OT *__restrict__ fxt_lo)
{
    const float ts = (float)(1 << TC_TW_LOG2);
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long nf = (long long)rows_pad * Kx_pad;
    if (idx < nf) {
        int n = (int)(idx / Kx_pad), x = (int)(idx % Kx_pad), k = n >> 1;
        float v = 0.f;
        if (k < nuv && x < N) {
            float2 f = fx[(size_t)k * N + x];
            v = ((n & 1) ? f.y : f.x) * ts;
        }
        if (fx8h) {
            if constexpr (sizeof(OT) == 2) {
                __half h;
                split_f8(v, F8_A_HI, F8_A_LO, h, fx8h[idx], fx8l[idx]);
                fx_hi[idx] = h;
            }
        } else {
            split_store(fx_hi, fx_lo, (size_t)idx, v);
        }
        return;
    }
    idx -= nf;
    if (idx < (long long)xrows_pad * K2_pad) {
        int x = (int)(idx / K2_pad), kp = (int)(idx % K2_pad), k = kp >> 1;
        float v = 0.f;
        if (k < nuv && x < N) {
            float2 f = fx[(size_t)k * N + x];
            v = ((kp & 1) ? f.y : f.x) * ts;
        }
        split_store(fxt_hi, fxt_lo, (size_t)idx, v);
    }
}

// Eight consecutive values of one operand row: hi (and lo) with 16-byte (f16)
// or 2 x 16-byte (TF32) stores.
template <typename OT>
__device__ __forceinline__ void split_store8(OT *__restrict__ hi, OT *__restrict__ lo, size_t off, const float (&v)[8])
{
    __align__(16) OT h[8];
    __align__(16) OT l[8];
#pragma unroll
    for (int j = 0; j < 8; j++) OpSplit<OT>::split(v[j], h[j], l[j]);
    constexpr int NV = sizeof(OT) * 8 / 16;
    uint4 *ph = reinterpret_cast<uint4 *>(hi + off);
#pragma unroll
    for (int k = 0; k < NV; k++) ph[k] = reinterpret_cast<const uint4 *>(h)[k];
    if (lo) {
        uint4 *pl = reinterpret_cast<uint4 *>(lo + off);
#pragma unroll
        for (int k = 0; k < NV; k++) pl[k] = reinterpret_cast<const uint4 *>(l)[k];
    }
}

// f16 operands: the same split with paired conversions
template <>
__device__ __forceinline__ void split_store8<__half>(__half *__restrict__ hi, __half *__restrict__ lo, size_t off,
                                                     const float (&v)[8])
{
    __align__(16) __half2 h[4];
    __align__(16) __half2 l[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        h[j] = __floats2half2_rn(v[2 * j], v[2 * j + 1]);
        const float2 b = __half22float2(h[j]);
        l[j] = __floats2half2_rn(v[2 * j] - b.x, v[2 * j + 1] - b.y);
    }
    *reinterpret_cast<uint4 *>(hi + off) = *reinterpret_cast<const uint4 *>(h);
    if (lo) *reinterpret_cast<uint4 *>(lo + off) = *reinterpret_cast<const uint4 *>(l);
}

__device__ __forceinline__ float warp_max_f(float v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, off));
    return v;
}


// Row-wise prep of the forward's image operand. A block of PR_THREADS threads
// works on R = 8 / W image rows at a time, W warps (a power of two) per row.
// (Narrow rows packed several to a warp, with a quarter of the blocks at 64²,
// measured slower in a 64-instance batch: 13.2 ms of trial prep against 11.3.)
//   MODE 0  the image as it is; with `reduce`, its flux, regulariser and max
//   MODE 1  the line-search trial I = max(I + s d, minval), s = cg.s, written to
//           dst, with its flux, regulariser and max
//   MODE 2  trial j (the grid's y) of a batched search, s = cg.ts[j], written to
//           dst + j npix and to operand rows j Lpad + y, with its flux and
//           regulariser; nothing when `gate` is set and *gate is 0
// Every row gets its own power-of-two scale 2^(15 - e), e the exponent of the
// row's max |I| (a reduction over the row's warps: no pass over the whole image
// has to end before the split), and the forward epilogue multiplies
// accumulator column y by rsc[row] = 2^(e - 15 - TC_TW_LOG2), exactly. With N a
// multiple of 8 and N <= 256 W every lane holds 8 consecutive pixels of its row
// in registers between the max and the split (16-byte loads and stores); other
// shapes take a scalar path that reads the row twice. Per-pixel regulariser
// terms in FP32 (reg_term_f); flux and regulariser are summed in FP64 in a
// fixed order (kernel_update_tempimage.cl, kernel_entropy_gs.cl;
// gpu.c:860-884).
#define PR_THREADS 256
#define PR_WARPS_MAX (PR_THREADS / 32)

// warps per image row: a power of two, at most PR_WARPS_MAX
static inline int pr_warps_per_row(int N)
{
    int w = 1;
    while (w < PR_WARPS_MAX && 256 * w < N) w <<= 1;
    return w;
}

struct PrepRowsArgs {
    const float *img, *d;
    float *dst;
    const float *model;
    int N, W, Lpad, Kx_pad;  // W warps per row
    void *hi, *lo;  // OT
    uint8_t *h8, *l8;
    float *rsc;
    int reduce;
    double *partials;
    DevScalars *sc;
    const int *gate;
    GP_VGRID_FIELDS;
};

template <typename OT, int MODE>
__device__ __forceinline__ void tc_prep_rows_body(const PrepRowsArgs &A, const GpVGrid &vg)
{
    const float *__restrict__ img = A.img;
    const float *__restrict__ d = A.d;
    float *__restrict__ dst = A.dst;
    const float *__restrict__ model = A.model;
    const int N = A.N, W = A.W, Lpad = A.Lpad, Kx_pad = A.Kx_pad, reduce = A.reduce;
    OT *__restrict__ hi = (OT *)A.hi;
    OT *__restrict__ lo = (OT *)A.lo;
    uint8_t *__restrict__ h8 = A.h8;
    uint8_t *__restrict__ l8 = A.l8;
    float *__restrict__ rsc = A.rsc;
    double *__restrict__ partials = A.partials;
    DevScalars *__restrict__ sc = A.sc;
    __shared__ double smem[3 * 32];
    __shared__ float wmax[PR_WARPS_MAX];
    if (A.gate && !*A.gate) return;  // lockstep batches: this instance's line search is over
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j = MODE == 2 ? vg.by : 0;
    const double s = MODE == 1 ? sc->cg.s : MODE == 2 ? sc->cg.ts[j] : 0.0;
    const double minval = MODE ? sc->cg.minvalue : 0.0;
    const int reg_kind = sc->reg_kind;
    const bool red = MODE ? true : reduce != 0;
    if (MODE == 2) dst += (size_t)j * N * N;
    const size_t row0 = (size_t)j * Lpad;
    const int R = PR_WARPS_MAX / W;            // rows per block and pass
    const int sub = warp % W, rw = warp / W;   // this warp's part of its row, row within the pass
    const int t = sub * 32 + lane, nt = 32 * W;  // thread within the row's group
    double acc[2] = {0.0, 0.0};
    float mx = 0.f;
    const bool vec = (N & 7) == 0 && N <= 8 * nt;
    // Trial images one warp wide (N <= 256): flux and regulariser summed per
    // image row into partials[j][y], then over the rows in a fixed order, so
    // the sums do not depend on the block grid (a staged batch gives a block
    // several passes). Wider rows: per-block partials.
    const bool rowsum = MODE == 2 && W == 1;
    double *__restrict__ rowp = partials + (size_t)j * N * 2;
    for (int ybase = vg.bx * R; ybase < N; ybase += vg.nbx * R) {  // block-uniform
        const int y = ybase + rw;
        const bool yv = y < N;
        const size_t rp = (size_t)(yv ? y : 0) * N;
        float rmax = 0.f;
        float v[8];
        const int x = 8 * t;
        const bool xv = vec && yv && x < N;
        if (vec) {
            if (xv) {
                *reinterpret_cast<float4 *>(&v[0]) = __ldg(reinterpret_cast<const float4 *>(img + rp + x));
                *reinterpret_cast<float4 *>(&v[4]) = __ldg(reinterpret_cast<const float4 *>(img + rp + x + 4));
                if (MODE) {
                    float dv[8];
                    *reinterpret_cast<float4 *>(&dv[0]) = __ldg(reinterpret_cast<const float4 *>(d + rp + x));
                    *reinterpret_cast<float4 *>(&dv[4]) = __ldg(reinterpret_cast<const float4 *>(d + rp + x + 4));
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        double tt = (double)v[k] + s * (double)dv[k];
                        if (tt < minval) tt = minval;
                        v[k] = (float)tt;
                    }
                    *reinterpret_cast<float4 *>(dst + rp + x) = *reinterpret_cast<const float4 *>(&v[0]);
                    *reinterpret_cast<float4 *>(dst + rp + x + 4) = *reinterpret_cast<const float4 *>(&v[4]);
                }
                if (red) {
                    float mv[8];
                    *reinterpret_cast<float4 *>(&mv[0]) = __ldg(reinterpret_cast<const float4 *>(model + rp + x));
                    *reinterpret_cast<float4 *>(&mv[4]) = __ldg(reinterpret_cast<const float4 *>(model + rp + x + 4));
#pragma unroll
                    for (int k = 0; k < 8; k++) acc[0] += (double)v[k];
                    reg_terms8(v, mv, reg_kind, acc[1]);
                }
#pragma unroll
                for (int k = 0; k < 8; k++) rmax = fmaxf(rmax, fabsf(v[k]));
            }
        } else if (yv) {
            for (int xx = t; xx < N; xx += nt) {
                float I = __ldg(&img[rp + xx]);
                if (MODE) {
                    double tt = (double)I + s * (double)__ldg(&d[rp + xx]);
                    if (tt < minval) tt = minval;
                    I = (float)tt;
                    dst[rp + xx] = I;
                }
                if (red) {
                    acc[0] += (double)I;
                    acc[1] += (double)reg_term_f(I, __ldg(&model[rp + xx]), reg_kind);
                }
                rmax = fmaxf(rmax, fabsf(I));
            }
        }
        // max over the row's W warps (one warp: the shuffle tree has it already)
        rmax = warp_max_f(rmax);
        if (W > 1) {  // block-uniform
            if (lane == 0) wmax[warp] = rmax;
            __syncthreads();
            rmax = 0.f;
            for (int q = 0; q < W; q++) rmax = fmaxf(rmax, wmax[rw * W + q]);
            __syncthreads();  // wmax is rewritten by the next pass
        }
        if (rowsum) {
            // this row's flux and regulariser, one fixed shuffle tree; lanes past
            // the row add +0.0
#pragma unroll
            for (int i = 0; i < 2; i++)
                for (int off = 16; off > 0; off >>= 1) acc[i] += __shfl_down_sync(0xffffffffu, acc[i], off);
            if (yv && lane == 0) {
                rowp[2 * y] = acc[0];
                rowp[2 * y + 1] = acc[1];
            }
            acc[0] = acc[1] = 0.0;
        }
        int ex = 0;
        frexpf(rmax, &ex);
        const float scale = ldexpf(1.f, 15 - ex);
        if (xv) {
#pragma unroll
            for (int k = 0; k < 8; k++) v[k] *= scale;
            const size_t o = (row0 + y) * Kx_pad + x;
            if (h8) {
                if constexpr (sizeof(OT) == 2) {
                    // f16 hi plus the E4M3 pair (hi / 2^10, lo * 4): 16 + 8 + 8 bytes
                    __align__(16) __half hh[8];
                    __align__(8) uint8_t qh[8], ql[8];
#pragma unroll
                    for (int k = 0; k < 8; k++) split_f8(v[k], F8_B_HI, F8_B_LO, hh[k], qh[k], ql[k]);
                    *reinterpret_cast<uint4 *>(hi + o) = *reinterpret_cast<const uint4 *>(hh);
                    *reinterpret_cast<uint2 *>(h8 + o) = *reinterpret_cast<const uint2 *>(qh);
                    *reinterpret_cast<uint2 *>(l8 + o) = *reinterpret_cast<const uint2 *>(ql);
                }
            } else {
                split_store8(hi, lo, o, v);
            }
        } else if (!vec && yv) {
            // second pass: each thread reads back the values it wrote (or the image)
            for (int xx = t; xx < N; xx += nt) {
                const float I = MODE ? dst[rp + xx] : __ldg(&img[rp + xx]);
                const size_t o = (row0 + y) * Kx_pad + xx;
                if (h8) {
                    if constexpr (sizeof(OT) == 2) {
                        __half hh;
                        split_f8(I * scale, F8_B_HI, F8_B_LO, hh, h8[o], l8[o]);
                        hi[o] = hh;
                    }
                } else {
                    split_store(hi, lo, o, I * scale);
                }
            }
        }
        if (yv && t == 0) rsc[row0 + y] = ldexpf(1.f, ex - 15 - TC_TW_LOG2);
        mx = fmaxf(mx, rmax);
    }
    if (!red) return;  // uniform over the grid
    if (MODE == 2) {
        double *pp = rowp;
        int np = N;
        if (!rowsum) {
            block_sum<2>(acc, smem);
            pp = partials + (size_t)j * vg.nbx * 2;
            np = vg.nbx;
            if (threadIdx.x == 0) {
                pp[2 * vg.bx] = acc[0];
                pp[2 * vg.bx + 1] = acc[1];
            }
        }
        if (last_block_of(&sc->t_counter[j], vg.nbx)) {
            double o[2];
            finish_sum<2>(pp, np, o, smem);
            if (threadIdx.x == 0) {
                sc->t_flux[j] = o[0];
                sc->t_invflux[j] = 1.0 / o[0];
                sc->t_entropy[j] = o[1];
                sc->t_counter[j] = 0;
            }
        }
        return;
    }
    block_sum<2>(acc, smem);
    const double bmax = block_max((double)mx, smem);
    if (threadIdx.x == 0) {
        partials[3 * vg.bx] = acc[0];
        partials[3 * vg.bx + 1] = acc[1];
        partials[3 * vg.bx + 2] = bmax;
    }
    if (last_block_of(&sc->counter[RED_PREP], vg.nbx)) {
        double v3[3];
        finish_sum<3>(partials, vg.nbx, v3, smem);
        // max over the blocks' maxima (any order gives the same value)
        double m = 0.0;
        for (int b = threadIdx.x; b < vg.nbx; b += blockDim.x) m = fmax(m, __ldcg(&partials[3 * b + 2]));
        m = block_max(m, smem);
        if (threadIdx.x == 0) {
            sc->flux = v3[0];
            sc->invflux = 1.0 / v3[0];
            sc->entropy = v3[1];
            sc->imax = m;
            sc->flux_f = (float)v3[0];
            sc->invflux_f = (float)(1.0 / v3[0]);
            sc->entropy_f = (float)v3[1];
            if (!isfinite(v3[0]) || !isfinite(v3[1])) sc->nonfinite |= 1u;
            sc->counter[RED_PREP] = 0;
        }
    }
}

template <typename OT, int MODE>
__global__ void __launch_bounds__(PR_THREADS) k_tc_prep_rows(const PrepRowsArgs a)
{
    gp_pdl_enter();
    tc_prep_rows_body<OT, MODE>(a, gp_vgrid_hw());
}

template <typename OT, int MODE> struct PrepRowsOp {
    using Args = PrepRowsArgs;
    static __device__ __forceinline__ void run(const Args &a, const GpVGrid &v) { tc_prep_rows_body<OT, MODE>(a, v); }
};

// Fy anchors every 16 image rows and the one-row rotation of every uv point
__global__ void k_tc_fy_anchors(const float2 *__restrict__ fy, int nuv, int N, int nanc, float2 *__restrict__ fya,
                                float2 *__restrict__ fyr)
{
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nuv * nanc) return;
    int k = (int)(idx / nanc), j = (int)(idx % nanc);
    fya[idx] = fy[(size_t)k * N + 16 * j];
    if (j == 0) fyr[k] = N > 1 ? fy[(size_t)k * N + 1] : make_float2(1.f, 0.f);
}

// Adjoint A operand W[y][2k+c] from c_k and Fy[k][y], one global power-of-two
// scale from max |c_k|; 32 uv x 32 rows per block, transposed through smem so
// that the writes of W are coalesced. Fy[k][y] = e^{-2 pi i s v_k y} is formed
// in place, as k_gen_twiddles forms the table (phase in turns in FP64, reduced
// to [-1/2, 1/2]) with the final sincos in FP32: the kernel reads no table and
// writes only W. Problems given as the reference's tables (no (u, v)) read Fy
// from the table instead (uvc == nullptr).
template <typename OT>
__global__ void __launch_bounds__(256) k_tc_build_w(const float2 *__restrict__ cw, const float2 *__restrict__ uvc,
                                                    const float2 *__restrict__ fy, float pix, int nuv, int N,
                                                    int K2_pad, OT *__restrict__ w_hi, OT *__restrict__ w_lo,
                                                    DevScalars *__restrict__ sc)
{
    __shared__ float2 tile[32][33];
    __shared__ double sv[32];
    __shared__ float2 cs[32];
    const double cmax = sc->cmax;
    int ex = 0;
    float wscale = 1.f;
    if (cmax > 0.0) {
        frexp(cmax * 1.4143, &ex);
        wscale = ldexpf(1.f, 15 - ex);
    }
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
        sc->gscale = 1.0 / ((double)wscale * (double)(1 << TC_TW_LOG2));
    const int k0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    if (threadIdx.x < 32) {
        const int k = k0 + threadIdx.x;
        sv[threadIdx.x] = (k < nuv && uvc) ? RPMAS_TC * (double)pix * (double)uvc[k].y : 0.0;
        cs[threadIdx.x] = k < nuv ? cw[k] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int j = ty; j < 32; j += 8) {
        int k = k0 + j, y = y0 + tx;
        float2 w = make_float2(0.f, 0.f);
        if (k < nuv && y < N) {
            float2 f;
            if (uvc) {
                double t = sv[j] * (double)y;
                t -= rint(t);
                float sn, cn;
                sincospif((float)(2.0 * t), &sn, &cn);
                f = make_float2(cn, -sn);
            } else {
                f = fy[(size_t)k * N + y];
            }
            const float2 c = cs[j];
            w = make_float2((c.x * f.x - c.y * f.y) * wscale, -(c.x * f.y + c.y * f.x) * wscale);
        }
        tile[j][tx] = w;  // [k][y]
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {
        int y = y0 + j;
        if (y >= N) continue;
        int kl = tx;  // one uv per thread: writes columns 2k, 2k+1
        int k = k0 + kl;
        if (2 * k + 1 >= K2_pad) continue;
        float2 w = tile[kl][j];
        split_store(w_hi, w_lo, (size_t)y * K2_pad + 2 * k, w.x);
        split_store(w_hi, w_lo, (size_t)y * K2_pad + 2 * k + 1, w.y);
    }
}

// The same W from the uv coordinates, without the transpose. A thread owns four
// consecutive uv points (columns 8g .. 8g+7: one 16-byte store per row into
// each of W hi and W lo, 512 contiguous bytes per warp) and BW_ROWS image rows.
// Fy[k][y] = e^{-2 pi i t_k y}, t_k = pix v_k in turns, is evaluated as
// A_k(y0) R_k(y - y0): the anchor A_k at every BW_SEG-th row and the
// rotations R_k(j) = e^{-2 pi i j t_k}, j < BW_SEG (a shared table: the eight
// warps of a block share their 128 uv points) both come from an FP64 phase
// reduced to [-1/2, 1/2] and FP32 sincospif, so every element is one complex
// product of two correctly rounded factors and no rounding error accumulates
// along y. Columns of uv points >= nuv (up to K2_pad) are written as zeros;
// rows >= N are not touched.
#define BW_SEG 8
#define BW_ROWS 16
struct BuildWArgs {
    const float2 *cw, *uvc;
    float pix;
    int nuv, N, K2_pad;
    void *w_hi, *w_lo;  // OT
    DevScalars *sc;
    GP_VGRID_FIELDS;
};

template <typename OT>
__device__ __forceinline__ void tc_build_w_uv_body(const BuildWArgs &A, const GpVGrid &vg)
{
    const float2 *__restrict__ cw = A.cw;
    const float2 *__restrict__ uvc = A.uvc;
    const float pix = A.pix;
    const int nuv = A.nuv, N = A.N, K2_pad = A.K2_pad;
    OT *__restrict__ w_hi = (OT *)A.w_hi;
    OT *__restrict__ w_lo = (OT *)A.w_lo;
    DevScalars *__restrict__ sc = A.sc;
    __shared__ __align__(16) float2 rp[BW_SEG][128];
    const double cmax = sc->cmax;
    int ex = 0;
    float wscale = 1.f;
    if (cmax > 0.0) {
        frexp(cmax * 1.4143, &ex);
        wscale = ldexpf(1.f, 15 - ex);
    }
    if (vg.bx == 0 && vg.by == 0 && threadIdx.x == 0)
        sc->gscale = 1.0 / ((double)wscale * (double)(1 << TC_TW_LOG2));
    const int kbase = vg.bx * 128;
    for (int e = threadIdx.x; e < BW_SEG * 128; e += blockDim.x) {
        const int j = e >> 7, k = kbase + (e & 127);
        float2 r = make_float2(1.f, 0.f);
        if (j > 0 && k < nuv) {
            double t = RPMAS_TC * (double)pix * (double)uvc[k].y * (double)j;
            t -= rint(t);
            float sn, cn;
            sincospif((float)(2.0 * t), &sn, &cn);
            r = make_float2(cn, -sn);
        }
        rp[j][e & 127] = r;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int g = vg.bx * 32 + lane;
    const int y0 = (vg.by * 8 + (threadIdx.x >> 5)) * BW_ROWS;
    if (8 * g >= K2_pad || y0 >= N) return;
    float2 cs[4], an[4];
    double tv[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int k = 4 * g + i;
        cs[i] = make_float2(0.f, 0.f);
        tv[i] = 0.0;
        if (k < nuv) {
            const float2 c = cw[k];
            cs[i] = make_float2(c.x * wscale, c.y * wscale);
            tv[i] = RPMAS_TC * (double)pix * (double)uvc[k].y;
        }
    }
    const int y1 = min(N, y0 + BW_ROWS);
    // 8 values per row and thread: one 16-byte store (f16) or two (TF32)
    constexpr int NV = sizeof(OT) * 8 / 16;
    uint4 *ph = reinterpret_cast<uint4 *>(w_hi + (size_t)y0 * K2_pad + 8 * g);
    uint4 *pl = w_lo ? reinterpret_cast<uint4 *>(w_lo + (size_t)y0 * K2_pad + 8 * g) : nullptr;
    const size_t step = (size_t)K2_pad * sizeof(OT) / 16;  // uint4 per row
    for (int y = y0; y < y1; y++) {
        const int j = (y - y0) & (BW_SEG - 1);
        if (j == 0) {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                double t = tv[i] * (double)y;
                t -= rint(t);
                float sn, cn;
                sincospif((float)(2.0 * t), &sn, &cn);
                an[i] = make_float2(cn, -sn);
            }
        }
        const float4 r01 = *reinterpret_cast<const float4 *>(&rp[j][4 * lane]);
        const float4 r23 = *reinterpret_cast<const float4 *>(&rp[j][4 * lane + 2]);
        const float2 r[4] = {make_float2(r01.x, r01.y), make_float2(r01.z, r01.w), make_float2(r23.x, r23.y),
                             make_float2(r23.z, r23.w)};
        __align__(16) OT hv[8];
        __align__(16) OT lv[8];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float2 f = make_float2(an[i].x * r[i].x - an[i].y * r[i].y, an[i].x * r[i].y + an[i].y * r[i].x);
            const float2 w = make_float2(cs[i].x * f.x - cs[i].y * f.y, -(cs[i].x * f.y + cs[i].y * f.x));
            OpSplit<OT>::split(w.x, hv[2 * i], lv[2 * i]);
            OpSplit<OT>::split(w.y, hv[2 * i + 1], lv[2 * i + 1]);
        }
#pragma unroll
        for (int v = 0; v < NV; v++) ph[v] = reinterpret_cast<const uint4 *>(hv)[v];
        ph += step;
        if (pl) {
#pragma unroll
            for (int v = 0; v < NV; v++) pl[v] = reinterpret_cast<const uint4 *>(lv)[v];
            pl += step;
        }
    }
}

template <typename OT>
__global__ void __launch_bounds__(256) k_tc_build_w_uv(const BuildWArgs a)
{
    gp_pdl_enter();
    tc_build_w_uv_body<OT>(a, gp_vgrid_hw());
}

template <typename OT> struct BuildWOp {
    using Args = BuildWArgs;
    static __device__ __forceinline__ void run(const Args &a, const GpVGrid &v) { tc_build_w_uv_body<OT>(a, v); }
};

// ------------------------------------------------------------ host side

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

static int tc_get_encode(gpair_ctx *c)
{
    if (g_encode) return GPAIR_OK;
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess
        || q != cudaDriverEntryPointSuccess || !fn) {
        snprintf(c->last_error, sizeof(c->last_error), "cuTensorMapEncodeTiled unavailable");
        return GPAIR_ERR_CUDA;
    }
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    return GPAIR_OK;
}

// 2-D operand tensor [rows][cols] (cols contiguous) of f16 (esz 2) or FP32/TF32
// (esz 4) elements; boxes of one 128-byte K-block row x box_rows, 128 B swizzle
static int tc_make_map(gpair_ctx *c, CUtensorMap *m, const void *base, long long rows, long long cols, int box_rows,
                       int esz)
{
    const int bk = TC_ROWB / esz;
    if (cols % bk || rows % box_rows || ((uintptr_t)base & 255)) {
        snprintf(c->last_error, sizeof(c->last_error), "tensor map shape/alignment violates TMA rules");
        return GPAIR_ERR_INVALID;
    }
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * esz};
    cuuint32_t box[2] = {(cuuint32_t)bk, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(m, esz == 2 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                          const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        snprintf(c->last_error, sizeof(c->last_error), "cuTensorMapEncodeTiled failed (%d)", (int)r);
        return GPAIR_ERR_CUDA;
    }
    return GPAIR_OK;
}

// operand kind and product count of a precision mode, and the forward's operand kind
static void tc_mode(int precision, int *op, int *nprod, int *fop = nullptr)
{
    *op = (precision == GPAIR_PREC_TF32 || precision == GPAIR_PREC_TF32X3) ? OP_TF32 : OP_F16;
    *nprod = precision == GPAIR_PREC_TF32 ? 1 : 3;
    if (fop) *fop = precision == GPAIR_PREC_SPLIT16F8 ? OP_F16F8 : *op;
}

// 2-D tensor [rows][cols] of bytes (E4M3), boxes of 64 bytes x box_rows, 64 B swizzle
static int tc_make_map8(gpair_ctx *c, CUtensorMap *m, const void *base, long long rows, long long cols, int box_rows)
{
    if (cols % 64 || rows % box_rows || ((uintptr_t)base & 255)) {
        snprintf(c->last_error, sizeof(c->last_error), "tensor map shape/alignment violates TMA rules");
        return GPAIR_ERR_INVALID;
    }
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols};
    cuuint32_t box[2] = {64u, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        snprintf(c->last_error, sizeof(c->last_error), "cuTensorMapEncodeTiled (8-bit) failed (%d)", (int)r);
        return GPAIR_ERR_CUDA;
    }
    return GPAIR_OK;
}

// Split-K of the tensor adjoint for K-blocks of `bk` elements: enough splits to
// fill the SMs, and at most TC_SPLIT_PRODUCTS products per split (FP32
// accumulation in TMEM: a running sum of n oscillating products carries a
// relative rounding error of about 2^-24 sqrt(n); 4096 keeps it near 4e-6; the
// splits are summed in FP64)
int gp_tc_splits(int N, int nuv, int nsm, int bk, int pair, int *kb_per_out)
{
    const int tm = pair ? 256 : TC_BM, slots = pair ? nsm / 2 : nsm;
    int M_pad = round_up(N, TC_BN), xrows_pad = round_up(N, tm), K2_pad = round_up(2LL * (nuv ? nuv : 1), bk);
    int tiles = (xrows_pad / tm) * (M_pad / TC_BN);
    int kb_total = K2_pad / bk;
    int want = (slots + tiles - 1) / tiles;
    if (want < 1) want = 1;
    if (want > kb_total) want = kb_total;
    int kb_per = (kb_total + want - 1) / want;
    const int cap = TC_SPLIT_PRODUCTS / bk;
    if (kb_per > cap) kb_per = cap;
    int splits = (kb_total + kb_per - 1) / kb_per;
    if (kb_per_out) *kb_per_out = kb_per;
    return splits;
}

// the largest split count any tensor mode uses for this shape
int gp_tc_max_splits(int N, int nuv, int nsm)
{
    int mx = 0;
    for (int op = OP_F16; op <= OP_TF32; op++)
        for (int pair = 0; pair <= 1; pair++) {
            const int v = gp_tc_splits(N, nuv, nsm, tc_bk(op), pair, nullptr);
            if (v > mx) mx = v;
        }
    return mx;
}

void gp_tc_free(gpair_ctx *c)
{
    TcState *t = (TcState *)c->tc_state;
    if (!t) return;
    c->buf_gen++;
    void *bufs[] = {t->img_hi, t->img_lo, t->fx_hi, t->fx_lo, t->fxt_hi, t->fxt_lo, t->w_hi, t->w_lo,
                    t->imgb_hi, t->imgb_lo, t->fx8h, t->fx8l, t->img8h, t->img8l, t->imgb8h, t->imgb8l};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (t->fya) cudaFree(t->fya);
    if (t->fyr) cudaFree(t->fyr);
    if (t->rsc) cudaFree(t->rsc);
    if (t->rscb) cudaFree(t->rscb);
    free(t);
    c->tc_state = nullptr;
}

template <typename OT>
static void launch_twiddle_ops(gpair_ctx *c, TcState *t, long long n_all)
{
    k_tc_twiddle_ops<OT><<<gp_cdiv(n_all, 256), 256, 0, c->stream>>>(
        c->fx, c->nuv, c->N, t->Kx_pad, t->rows_pad, t->K2_pad, t->xrows_pad, (OT *)t->fx_hi, (OT *)t->fx_lo,
        (uint8_t *)t->fx8h, (uint8_t *)t->fx8l, (OT *)t->fxt_hi, (OT *)t->fxt_lo);
}

template <int EPI, int PAIR, int GROUP>
static int tc_set_smem(gpair_ctx *c)
{
    const int bytes = GROUP ? TC_SMEM_GROUP_BYTES : TC_SMEM_BYTES;
    GP_CUDA(c, cudaFuncSetAttribute(k_tc_gemm<EPI, OP_F16, 3, PAIR, GROUP>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    GP_CUDA(c, cudaFuncSetAttribute(k_tc_gemm<EPI, OP_TF32, 3, PAIR, GROUP>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    GP_CUDA(c, cudaFuncSetAttribute(k_tc_gemm<EPI, OP_TF32, 1, PAIR, GROUP>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    if (EPI == EPI_FWD)
        GP_CUDA(c, cudaFuncSetAttribute(k_tc_gemm<EPI_FWD, OP_F16F8, 3, PAIR, GROUP>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    return GPAIR_OK;
}

int gp_tc_prepare(gpair_ctx *c)
{
    if (!c->have_problem) return GPAIR_OK;  // prepared when the problem is loaded
    int op, nprod, fop;
    tc_mode(c->precision, &op, &nprod, &fop);
    const int pair = c->tc_pair ? 1 : 0;
    TcState *old = (TcState *)c->tc_state;
    if (old && old->op == op && old->nprod == nprod && old->fop == fop && old->pair == pair) return GPAIR_OK;
    if (old) {
        // another operand kind: rebuild every operand buffer for this mode
        GP_CUDA(c, cudaStreamSynchronize(c->stream));
        gp_tc_free(c);
    }
    int rc = tc_get_encode(c);
    if (rc) return rc;
    TcState *t = (TcState *)calloc(1, sizeof(TcState));
    if (!t) return GPAIR_ERR_ALLOC;
    c->tc_state = t;
    t->op = op;
    t->nprod = nprod;
    t->fop = fop;
    t->pair = pair;
    t->esz = op == OP_F16 ? 2 : 4;
    t->bk = tc_bk(op);
    const int N = c->N, nuv = c->nuv ? c->nuv : 1;
    t->Kx_pad = round_up(N, t->bk);
    t->M_pad = round_up(N, TC_BN);
    const int tm = pair ? 256 : TC_BM;  // A rows per tile
    t->rows_pad = round_up(2LL * nuv, tm);
    t->K2_pad = round_up(2LL * nuv, t->bk);
    t->xrows_pad = round_up(N, tm);
    GP_CUDA(c, cudaDeviceGetAttribute(&t->nsm, cudaDevAttrMultiProcessorCount, c->device));
    t->splits = gp_tc_splits(N, nuv, t->nsm, t->bk, pair, &t->kb_per);
    size_t img = (size_t)t->M_pad * t->Kx_pad, fxs = (size_t)t->rows_pad * t->Kx_pad;
    size_t fxts = (size_t)t->xrows_pad * t->K2_pad, ws = (size_t)t->M_pad * t->K2_pad;
    const bool f8 = fop == OP_F16F8;
    // f8: the forward's lo operands are E4M3 pairs (1 byte per element each)
    struct { void **p; size_t n; bool lo; int esz; } al[] = {
        {&t->img_hi, img, false, t->esz},  {&t->img_lo, f8 ? 0 : img, true, t->esz},
        {&t->fx_hi, fxs, false, t->esz},   {&t->fx_lo, f8 ? 0 : fxs, true, t->esz},
        {&t->fxt_hi, fxts, false, t->esz}, {&t->fxt_lo, fxts, true, t->esz},
        {&t->w_hi, ws, false, t->esz},     {&t->w_lo, ws, true, t->esz},
        {&t->img8h, f8 ? img : 0, true, 1}, {&t->img8l, f8 ? img : 0, true, 1},
        {&t->fx8h, f8 ? fxs : 0, true, 1},  {&t->fx8l, f8 ? fxs : 0, true, 1}};
    for (auto &x : al) {
        if ((x.lo && nprod == 1) || x.n == 0) continue;  // one product: no lo operands
        GP_CUDA(c, cudaMalloc(x.p, x.n * x.esz));
        GP_CUDA(c, cudaMemsetAsync(*x.p, 0, x.n * x.esz, c->stream));
    }
    GP_CUDA(c, cudaMalloc(&t->rsc, sizeof(float) * (size_t)t->M_pad));
    GP_CUDA(c, cudaMemsetAsync(t->rsc, 0, sizeof(float) * (size_t)t->M_pad, c->stream));
    t->nanc = (N + 15) / 16;
    GP_CUDA(c, cudaMalloc(&t->fya, sizeof(float2) * (size_t)nuv * t->nanc));
    GP_CUDA(c, cudaMalloc(&t->fyr, sizeof(float2) * (size_t)nuv));
    if (c->nuv) {
        k_tc_fy_anchors<<<gp_cdiv((long long)c->nuv * t->nanc, 256), 256, 0, c->stream>>>(c->fy, c->nuv, N, t->nanc,
                                                                                         t->fya, t->fyr);
        GP_LAUNCH_CHECK(c);
    }
    long long n_all = (long long)fxs + (long long)fxts;
    if (op == OP_F16) launch_twiddle_ops<__half>(c, t, n_all);
    else launch_twiddle_ops<float>(c, t, n_all);
    GP_LAUNCH_CHECK(c);
    const int e = t->esz;
    const int bbox = pair ? 128 : TC_BN;  // B rows one CTA stages
    if ((rc = tc_make_map(c, &t->m_img_hi, t->img_hi, t->M_pad, t->Kx_pad, bbox, e))) return rc;
    if ((rc = tc_make_map(c, &t->m_fx_hi, t->fx_hi, t->rows_pad, t->Kx_pad, TC_BM, e))) return rc;
    if ((rc = tc_make_map(c, &t->m_w_hi, t->w_hi, t->M_pad, t->K2_pad, bbox, e))) return rc;
    if ((rc = tc_make_map(c, &t->m_fxt_hi, t->fxt_hi, t->xrows_pad, t->K2_pad, TC_BM, e))) return rc;
    if (nprod == 3) {
        if (f8) {
            if ((rc = tc_make_map8(c, &t->m_img8h, t->img8h, t->M_pad, t->Kx_pad, bbox))) return rc;
            if ((rc = tc_make_map8(c, &t->m_img8l, t->img8l, t->M_pad, t->Kx_pad, bbox))) return rc;
            if ((rc = tc_make_map8(c, &t->m_fx8h, t->fx8h, t->rows_pad, t->Kx_pad, TC_BM))) return rc;
            if ((rc = tc_make_map8(c, &t->m_fx8l, t->fx8l, t->rows_pad, t->Kx_pad, TC_BM))) return rc;
            t->m_img_lo = t->m_img_hi;  // not loaded by the OP_F16F8 forward
            t->m_fx_lo = t->m_fx_hi;
        } else {
            if ((rc = tc_make_map(c, &t->m_img_lo, t->img_lo, t->M_pad, t->Kx_pad, bbox, e))) return rc;
            if ((rc = tc_make_map(c, &t->m_fx_lo, t->fx_lo, t->rows_pad, t->Kx_pad, TC_BM, e))) return rc;
        }
        if ((rc = tc_make_map(c, &t->m_w_lo, t->w_lo, t->M_pad, t->K2_pad, bbox, e))) return rc;
        if ((rc = tc_make_map(c, &t->m_fxt_lo, t->fxt_lo, t->xrows_pad, t->K2_pad, TC_BM, e))) return rc;
    } else {
        // the kernel never loads the lo maps in one-product mode; pass valid maps anyway
        t->m_img_lo = t->m_img_hi;
        t->m_fx_lo = t->m_fx_hi;
        t->m_w_lo = t->m_w_hi;
        t->m_fxt_lo = t->m_fxt_hi;
    }
    if ((rc = tc_set_smem<EPI_FWD, 0, 0>(c))) return rc;
    if ((rc = tc_set_smem<EPI_STORE, 0, 0>(c))) return rc;
    if ((rc = tc_set_smem<EPI_FWD, 1, 0>(c))) return rc;
    if ((rc = tc_set_smem<EPI_STORE, 1, 0>(c))) return rc;
    if ((rc = tc_set_smem<EPI_FWD, 0, 1>(c))) return rc;
    if ((rc = tc_set_smem<EPI_FWD, 1, 1>(c))) return rc;
    if ((rc = tc_set_smem<EPI_STORE, 0, 1>(c))) return rc;
    if ((rc = tc_set_smem<EPI_STORE, 1, 1>(c))) return rc;
    t->npairs = t->nsm / 2;
    if (pair) {
        // clusters of two that can be resident at once (an SM left over in a GPC cannot host a pair)
        cudaLaunchConfig_t cfg;
        memset(&cfg, 0, sizeof(cfg));
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 2;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(2 * (unsigned)t->npairs, 1, 1);
        cfg.blockDim = dim3(tc_threads<EPI_FWD>(), 1, 1);
        cfg.dynamicSmemBytes = TC_SMEM_BYTES;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, (const void *)k_tc_gemm<EPI_FWD, OP_F16, 3, 1, 0>, &cfg) ==
                cudaSuccess &&
            nclusters > 0 && nclusters < t->npairs)
            t->npairs = nclusters;
        cudaGetLastError();
    }
    GP_CUDA(c, cudaStreamSynchronize(c->stream));
    return GPAIR_OK;
}

// split-K tile length of the tensor adjoint (K-blocks per split): read / override
int gp_tc_kb_per(gpair_ctx *c)
{
    TcState *t = (TcState *)c->tc_state;
    return t ? t->kb_per : 0;
}

// split count of the tensor adjoint for a given split-K tile length
int gp_tc_split_count(gpair_ctx *c, int kb_per)
{
    TcState *t = (TcState *)c->tc_state;
    if (!t || kb_per <= 0) return 0;
    return (t->K2_pad / t->bk + kb_per - 1) / kb_per;
}

// the largest split-K tile length the FP32 accumulation allows
int gp_tc_kb_cap(gpair_ctx *c)
{
    TcState *t = (TcState *)c->tc_state;
    return t ? TC_SPLIT_PRODUCTS / t->bk : 0;
}

int gp_tc_set_kb_per(gpair_ctx *c, int kb_per)
{
    TcState *t = (TcState *)c->tc_state;
    if (!t) return GPAIR_ERR_STATE;
    const int kb_total = t->K2_pad / t->bk;
    if (kb_per < 1 || kb_per > TC_SPLIT_PRODUCTS / t->bk) return GPAIR_ERR_INVALID;
    const int splits = (kb_total + kb_per - 1) / kb_per;
    if (splits > c->gpart_cap) return GPAIR_ERR_INVALID;
    t->kb_per = kb_per;
    t->splits = splits;
    return GPAIR_OK;
}

// Split-K lengths for n contexts that share the GPU (concurrent runs, batches):
// their adjoint units together fill the SMs about twice, each context's share
// in proportion to its adjoint work, instead of each filling the GPU alone.
// Longer splits mean fewer partial images to write in the adjoint and to sum
// in the gradient. Captured CG graphs of a changed context are dropped.
static TcState *tc_state_ready(gpair_ctx *c, int *rc);

int gp_tc_shared_splits(gpair_ctx **ctx, int n)
{
    if (!ctx || n < 1) return GPAIR_ERR_INVALID;
    double total = 0.0;
    int slots = 0;
    for (int i = 0; i < n; i++) {
        if (!ctx[i] || !ctx[i]->have_problem) return GPAIR_ERR_STATE;
        if (ctx[i]->precision == GPAIR_PREC_FP32) continue;
        int rc;
        TcState *t = tc_state_ready(ctx[i], &rc);
        if (rc) return rc;
        const int tiles = (t->xrows_pad / (t->pair ? 256 : TC_BM)) * (t->M_pad / TC_BN);
        total += (double)tiles * (double)(t->K2_pad / t->bk);
        if (!slots) slots = t->pair ? t->npairs : t->nsm;
    }
    for (int i = 0; i < n; i++)
        if (ctx[i]->gf_parts != 1) {
            ctx[i]->gf_parts = 1;  // one thread per four pixels in the gradient's split sum
            gp_cg_graph_free(ctx[i]);
        }
    if (total <= 0.0) return GPAIR_OK;
    const double target = 2.0 * slots;  // units over all contexts
    for (int i = 0; i < n; i++) {
        gpair_ctx *c = ctx[i];
        if (c->precision == GPAIR_PREC_FP32) continue;
        TcState *t = (TcState *)c->tc_state;
        const int kb_total = t->K2_pad / t->bk;
        int want = (int)(target * (double)kb_total / total + 0.5);  // splits of this context
        if (want < 1) want = 1;
        if (want > kb_total) want = kb_total;
        int kb_per = (kb_total + want - 1) / want;
        const int cap = TC_SPLIT_PRODUCTS / t->bk;
        if (kb_per > cap) kb_per = cap;
        if (kb_per != t->kb_per) {
            int rc = gp_tc_set_kb_per(c, kb_per);
            if (rc) return rc;
            gp_cg_graph_free(c);  // a captured CG graph holds the old split count
        }
    }
    return GPAIR_OK;
}

static TcState *tc_state_ready(gpair_ctx *c, int *rc)
{
    TcState *t = (TcState *)c->tc_state;
    *rc = GPAIR_OK;
    if (!t) {
        *rc = gp_tc_prepare(c);
        t = (TcState *)c->tc_state;
        if (!*rc && !t) *rc = GPAIR_ERR_STATE;
    }
    return t;
}

// The maps of one contraction: (A_hi, A_lo, A_x, B_hi, B_lo, B_x); A_x and B_x
// are read by the OP_F16F8 forward only
struct TcMaps {
    const CUtensorMap *a_hi, *a_lo, *a_x, *b_hi, *b_lo, *b_x;
};

// launch attributes of a contraction: the cluster of a CTA pair and the
// programmatic dependent launch (gp_launch)
static int tc_attrs(cudaLaunchAttribute *at, int pair, int pdl)
{
    int n = 0;
    if (pair) {
        at[n].id = cudaLaunchAttributeClusterDimension;
        at[n].val.clusterDim.x = 2;
        at[n].val.clusterDim.y = 1;
        at[n].val.clusterDim.z = 1;
        n++;
    }
    if (pdl) {
        at[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[n].val.programmaticStreamSerializationAllowed = 1;
        n++;
    }
    return n;
}

template <int EPI, int PAIR>
static cudaError_t tc_launch_kind(TcState *t, dim3 grid, cudaStream_t st, int pdl, const TcMaps &m, const TcArgs &a)
{
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cudaLaunchAttribute at[2];
    cfg.gridDim = grid;
    cfg.blockDim = dim3(tc_threads<EPI>(), 1, 1);
    cfg.dynamicSmemBytes = TC_SMEM_BYTES;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = tc_attrs(at, PAIR, pdl);
    if (EPI == EPI_FWD && t->fop == OP_F16F8)
        return cudaLaunchKernelEx(&cfg, k_tc_gemm<EPI_FWD, OP_F16F8, 3, PAIR, 0>, *m.a_hi, *m.a_lo, *m.a_x, *m.b_hi,
                                  *m.b_lo, *m.b_x, a);
    if (t->op == OP_F16)
        return cudaLaunchKernelEx(&cfg, k_tc_gemm<EPI, OP_F16, 3, PAIR, 0>, *m.a_hi, *m.a_lo, *m.a_x, *m.b_hi,
                                  *m.b_lo, *m.b_x, a);
    if (t->nprod == 3)
        return cudaLaunchKernelEx(&cfg, k_tc_gemm<EPI, OP_TF32, 3, PAIR, 0>, *m.a_hi, *m.a_lo, *m.a_x, *m.b_hi,
                                  *m.b_lo, *m.b_x, a);
    return cudaLaunchKernelEx(&cfg, k_tc_gemm<EPI, OP_TF32, 1, PAIR, 0>, *m.a_hi, *m.a_lo, *m.a_x, *m.b_hi,
                              *m.b_lo, *m.b_x, a);
}

// one launch of the contraction in the context's operand kind / product count:
// persistent CTAs (or CTA pairs), one per SM (pair of SMs) at most
template <int EPI>
static int tc_launch(gpair_ctx *c, TcState *t, const TcMaps &m, TcArgs &a)
{
    a.err = &c->sc->tc_err;
    a.budget = c->tc_wait_budget > 0 ? c->tc_wait_budget : TC_WAIT_BUDGET;
    a.skip_loads = c->tc_skip_loads;
    cudaError_t e;
    if (t->pair) {
        const int np = a.units < t->npairs ? a.units : t->npairs;
        e = tc_launch_kind<EPI, 1>(t, dim3(2 * np, 1, 1), c->stream, c->pdl, m, a);
    } else {
        const int g = a.units < t->nsm ? a.units : t->nsm;
        e = tc_launch_kind<EPI, 0>(t, dim3(g, 1, 1), c->stream, c->pdl, m, a);
    }
    if (e != cudaSuccess) {
        snprintf(c->last_error, sizeof(c->last_error), "tensor-core contraction launch: %s", cudaGetErrorString(e));
        return GPAIR_ERR_CUDA;
    }
    c->launches++;
    return GPAIR_OK;
}

// the forward's maps over an image-side operand (single image or batch stack)
static TcMaps tc_fwd_maps(const TcState *t, bool batch)
{
    const bool f8 = t->fop == OP_F16F8;
    TcMaps m;
    m.a_hi = &t->m_fx_hi;
    m.a_lo = f8 ? &t->m_fx8h : &t->m_fx_lo;
    m.a_x = f8 ? &t->m_fx8l : &t->m_fx_hi;
    m.b_hi = batch ? &t->m_imgb_hi : &t->m_img_hi;
    m.b_lo = f8 ? (batch ? &t->m_imgb8h : &t->m_img8h) : (batch ? &t->m_imgb_lo : &t->m_img_lo);
    m.b_x = f8 ? (batch ? &t->m_imgb8l : &t->m_img8l) : m.b_hi;
    return m;
}

// Row-wise prep launches (k_tc_prep_rows): PR_THREADS threads per block, R rows
// per block and pass; at most GP_MAX_PARTIALS blocks (three partials each fit
// the RED_PREP slot), a batch at most 1024 per trial (two partials each).
static PrepRowsArgs tc_prep_rows_args(gpair_ctx *c, TcState *t, int mode, int reduce, double *partials,
                                      const float *img)
{
    const int W = pr_warps_per_row(c->N), R = PR_WARPS_MAX / W;
    int gx = gp_cdiv(c->N, R);
    const int cap = mode == 2 ? 1024 : GP_MAX_PARTIALS;
    if (gx > cap) gx = cap;
    if (gx < 1) gx = 1;
    const bool b = mode == 2;
    PrepRowsArgs a;
    memset(&a, 0, sizeof(a));
    a.img = mode == 0 ? img : c->image;
    a.d = c->descent_dir;
    a.dst = mode == 1 ? c->image_temp : mode == 2 ? c->image_trials : nullptr;
    a.model = c->model;
    a.N = c->N;
    a.W = W;
    a.Lpad = b ? t->Lb : 0;
    a.Kx_pad = t->Kx_pad;
    a.hi = b ? t->imgb_hi : t->img_hi;
    a.lo = b ? t->imgb_lo : t->img_lo;
    a.h8 = (uint8_t *)(b ? t->imgb8h : t->img8h);
    a.l8 = (uint8_t *)(b ? t->imgb8l : t->img8l);
    a.rsc = b ? t->rscb : t->rsc;
    a.reduce = mode ? 1 : reduce;
    a.partials = partials;
    a.sc = c->sc;
    a.gate = b ? c->gate : nullptr;
    a.nbx = gx;
    a.nby = b ? GP_NTR : 1;
    return a;
}

static int tc_prep_rows_launch(gpair_ctx *c, TcState *t, int mode, int reduce, double *partials,
                               const float *img = nullptr)
{
    const PrepRowsArgs a = tc_prep_rows_args(c, t, mode, reduce, partials, img);
    const dim3 g(a.nbx, a.nby, 1), b(PR_THREADS);
    const bool f16 = t->op == OP_F16;
    if (mode == 0)
        GP_LAUNCH(c, gp_launch(c, f16 ? k_tc_prep_rows<__half, 0> : k_tc_prep_rows<float, 0>, g, b, 0, a));
    else if (mode == 1)
        GP_LAUNCH(c, gp_launch(c, f16 ? k_tc_prep_rows<__half, 1> : k_tc_prep_rows<float, 1>, g, b, 0, a));
    else
        GP_LAUNCH(c, gp_launch(c, f16 ? k_tc_prep_rows<__half, 2> : k_tc_prep_rows<float, 2>, g, b, 0, a));
    return GPAIR_OK;
}

// forward contraction on the already split image operand
int gp_tc_forward_gemm(gpair_ctx *c)
{
    int rc;
    TcState *t = tc_state_ready(c, &rc);
    if (rc) return rc;
    TcArgs a;
    memset(&a, 0, sizeof(a));
    a.m_tiles = t->rows_pad / (t->pair ? 256 : TC_BM);  // twiddle-row tiles
    a.n_tiles = t->M_pad / TC_BN;     // image-row tiles
    a.kb_total = t->Kx_pad / t->bk;
    a.kb_per_split = a.kb_total;
    a.units = a.m_tiles * a.n_tiles;
    a.fya = t->fya;
    a.fyr = t->fyr;
    a.nanc = t->nanc;
    a.N = c->N;
    a.nuv = c->nuv;
    a.lpad = t->M_pad;  // one image, partial entries of TC_EPI_COLS rows (one epilogue warp's columns)
    a.elog2 = 7;
    a.rsc = t->rsc;
    a.vpart = c->vpart;
    if ((rc = tc_launch<EPI_FWD>(c, t, tc_fwd_maps(t, false), a))) return rc;
    c->mt = t->M_pad / TC_EPI_COLS;
    return GPAIR_OK;
}

// Operand stack of the batched line-search trials: GP_NTR images of Lb rows
// (Lb = 32, 64 or 128 for small images so that 256-row tiles hold several
// whole images, else N rounded up to 256); partial entries of min(Lb, 256) rows.
int gp_tc_batch_prepare(gpair_ctx *c, int *epp)
{
    int rc;
    TcState *t = tc_state_ready(c, &rc);
    if (rc) return rc;
    if (!t->imgb_hi) {
        const int N = c->N;
        t->Lb = N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : round_up(N, TC_BN);
        const int erows = t->Lb < TC_EPI_COLS ? t->Lb : TC_EPI_COLS;
        t->epp_b = t->Lb / erows;
        const size_t rows = (size_t)GP_NTR * t->Lb, n = rows * t->Kx_pad;
        GP_CUDA(c, cudaMalloc(&t->rscb, sizeof(float) * rows));
        GP_CUDA(c, cudaMemsetAsync(t->rscb, 0, sizeof(float) * rows, c->stream));
        GP_CUDA(c, cudaMalloc(&t->imgb_hi, n * t->esz));
        GP_CUDA(c, cudaMemsetAsync(t->imgb_hi, 0, n * t->esz, c->stream));
        const int bbox = t->pair ? 128 : TC_BN;
        if ((rc = tc_make_map(c, &t->m_imgb_hi, t->imgb_hi, (long long)rows, t->Kx_pad, bbox, t->esz))) return rc;
        if (t->fop == OP_F16F8) {
            GP_CUDA(c, cudaMalloc(&t->imgb8h, n));
            GP_CUDA(c, cudaMemsetAsync(t->imgb8h, 0, n, c->stream));
            GP_CUDA(c, cudaMalloc(&t->imgb8l, n));
            GP_CUDA(c, cudaMemsetAsync(t->imgb8l, 0, n, c->stream));
            if ((rc = tc_make_map8(c, &t->m_imgb8h, t->imgb8h, (long long)rows, t->Kx_pad, bbox))) return rc;
            if ((rc = tc_make_map8(c, &t->m_imgb8l, t->imgb8l, (long long)rows, t->Kx_pad, bbox))) return rc;
            t->m_imgb_lo = t->m_imgb_hi;  // not loaded by the OP_F16F8 forward
        } else if (t->nprod == 3) {
            GP_CUDA(c, cudaMalloc(&t->imgb_lo, n * t->esz));
            GP_CUDA(c, cudaMemsetAsync(t->imgb_lo, 0, n * t->esz, c->stream));
            if ((rc = tc_make_map(c, &t->m_imgb_lo, t->imgb_lo, (long long)rows, t->Kx_pad, bbox, t->esz)))
                return rc;
        } else {
            t->m_imgb_lo = t->m_imgb_hi;
        }
    }
    c->epp = t->epp_b;
    if (epp) *epp = t->epp_b;
    return GPAIR_OK;
}

// trial images + their operands for a batch (steps from the device state)
int gp_tc_trials_prep_split(gpair_ctx *c, double *partials)
{
    int rc;
    TcState *t = tc_state_ready(c, &rc);
    if (rc) return rc;
    if ((rc = gp_tc_batch_prepare(c, nullptr))) return rc;
    return tc_prep_rows_launch(c, t, 2, 1, partials);
}

// forward contraction of the GP_NTR trial images in one launch: every twiddle
// tile is loaded once for the whole batch
int gp_tc_forward_batch_gemm(gpair_ctx *c)
{
    int rc;
    TcState *t = tc_state_ready(c, &rc);
    if (rc) return rc;
    if ((rc = gp_tc_batch_prepare(c, nullptr))) return rc;
    TcArgs a;
    memset(&a, 0, sizeof(a));
    a.m_tiles = t->rows_pad / (t->pair ? 256 : TC_BM);
    a.n_tiles = (GP_NTR * t->Lb) / TC_BN;
    a.kb_total = t->Kx_pad / t->bk;
    a.kb_per_split = a.kb_total;
    a.units = a.m_tiles * a.n_tiles;
    a.fya = t->fya;
    a.fyr = t->fyr;
    a.nanc = t->nanc;
    a.N = c->N;
    a.nuv = c->nuv;
    a.lpad = t->Lb;
    const int erows = t->Lb < TC_EPI_COLS ? t->Lb : TC_EPI_COLS;
    a.elog2 = erows == 32 ? 5 : erows == 64 ? 6 : 7;
    a.rsc = t->rscb;
    a.vpart = c->vpart_b;
    return tc_launch<EPI_FWD>(c, t, tc_fwd_maps(t, true), a);
}

// split of an image into the forward's image operand (its flux and regulariser
// already reduced)
int gp_tc_split(gpair_ctx *c, int which)
{
    int rc;
    TcState *t = tc_state_ready(c, &rc);
    if (rc) return rc;
    return tc_prep_rows_launch(c, t, 0, 0, nullptr, which == GPAIR_IMG_TEMP ? c->image_temp : c->image);
}

int gp_tc_forward(gpair_ctx *c, int which)
{
    int rc = gp_tc_split(c, which);
    if (rc) return rc;
    return gp_tc_forward_gemm(c);
}

// flux, regulariser and max of an image, and its forward operand, in one pass
int gp_tc_prep_image(gpair_ctx *c, int which)
{
    int rc;
    TcState *t = tc_state_ready(c, &rc);
    if (rc) return rc;
    return tc_prep_rows_launch(c, t, 0, 1, c->partials, which == GPAIR_IMG_TEMP ? c->image_temp : c->image);
}

// trial image + split in one kernel (reads s and minval from the device state)
int gp_tc_prep_split_trial(gpair_ctx *c)
{
    int rc;
    TcState *t = tc_state_ready(c, &rc);
    if (rc) return rc;
    return tc_prep_rows_launch(c, t, 1, 1, c->partials);
}

// 32 groups of 4 uv points x 8 warps of BW_ROWS rows per block
static BuildWArgs tc_build_w_args(gpair_ctx *c, TcState *t)
{
    BuildWArgs a = {c->cw, c->uvc, c->pix, c->nuv, c->N, t->K2_pad, t->w_hi, t->w_lo, c->sc,
                    gp_cdiv(t->K2_pad / 8, 32), gp_cdiv(c->N, 8 * BW_ROWS)};
    return a;
}

template <typename OT>
static cudaError_t launch_build_w(gpair_ctx *c, TcState *t)
{
    if (c->have_uv) {
        const BuildWArgs a = tc_build_w_args(c, t);
        return gp_launch(c, k_tc_build_w_uv<OT>, dim3(a.nbx, a.nby), dim3(256), 0, a);
    }
    dim3 g(gp_cdiv(c->nuv ? c->nuv : 1, 32), gp_cdiv(c->N, 32));
    k_tc_build_w<OT><<<g, 256, 0, c->stream>>>(c->cw, nullptr, c->fy, c->pix, c->nuv, c->N, t->K2_pad,
                                                (OT *)t->w_hi, (OT *)t->w_lo, c->sc);
    return cudaSuccess;
}

// adjoint A-side weights W from c_k and Fy (hi/lo, one global scale)
int gp_tc_build_w(gpair_ctx *c)
{
    int rc;
    TcState *t = tc_state_ready(c, &rc);
    if (rc) return rc;
    GP_LAUNCH(c, t->op == OP_F16 ? launch_build_w<__half>(c, t) : launch_build_w<float>(c, t));
    return GPAIR_OK;
}

// adjoint contraction on the already built weights: S split-K partial images
int gp_tc_adjoint_gemm(gpair_ctx *c)
{
    int rc;
    TcState *t = tc_state_ready(c, &rc);
    if (rc) return rc;
    TcArgs a;
    memset(&a, 0, sizeof(a));
    a.m_tiles = t->xrows_pad / (t->pair ? 256 : TC_BM);  // image-column tiles (twiddle side)
    a.n_tiles = t->M_pad / TC_BN;      // image-row tiles (weight side)
    a.kb_total = t->K2_pad / t->bk;
    a.kb_per_split = t->kb_per;
    a.units = a.m_tiles * a.n_tiles * t->splits;
    a.gpart = c->gpart;
    a.out_ld = c->N;
    a.out_rows = c->N;
    a.out_cols = c->N;
    const TcMaps m = {&t->m_fxt_hi, &t->m_fxt_lo, &t->m_fxt_hi, &t->m_w_hi, &t->m_w_lo, &t->m_w_hi};
    if ((rc = tc_launch<EPI_STORE>(c, t, m, a))) return rc;
    c->splits = t->splits;
    return GPAIR_OK;
}

int gp_tc_adjoint(gpair_ctx *c, int which)
{
    (void)which;
    int rc = gp_tc_build_w(c);
    if (rc) return rc;
    return gp_tc_adjoint_gemm(c);
}

// ------------------------------------------------------ grouped forward
//
// One tcgen05 launch over the batched-trial forwards of several instances
// (many independent reconstructions advancing in lockstep): the units of every
// gated instance, each with its own maps and epilogue arguments from a
// TcGroupInst array in global memory, share the persistent CTAs (or CTA pairs).
// All instances use the same operand kind, product count and tile layout.
struct TcGroup {
    int n, epi, op, nprod, pair, npairs, nsm;  // op: the operand kind of the contraction (the forward's: fop)
    TcGroupInst *d_inst;  // [n], device
    CUtensorMap map0;     // a valid map for the kernel's unused map parameters
    const int *gate;      // [n], device, owned by the caller
    unsigned int *err;    // bounded-wait failures of the grouped launches (device word of the caller)
};

void gp_tc_group_free(void *grp)
{
    TcGroup *G = (TcGroup *)grp;
    if (!G) return;
    if (G->d_inst) cudaFree(G->d_inst);
    free(G);
}

// the tile layout, operand kind, product count and forward operand kind of a
// context's tensor path (instances with equal keys can share a grouped forward;
// with equal key >> 3 -- all but the forward operand kind -- a grouped adjoint),
// or -1 on the CUDA cores. Sorting by key keeps both kinds of class contiguous.
int gp_tc_group_key(gpair_ctx *c)
{
    if (c->precision == GPAIR_PREC_FP32) return -1;
    int op, nprod, fop;
    tc_mode(c->precision, &op, &nprod, &fop);
    return (((c->tc_pair ? 1 : 0) * 8 + op) * 4 + nprod) * 8 + fop;
}

// one instance's entry of a grouped contraction of kind GP_TCG_*
static void tc_group_inst(gpair_ctx *c, TcState *t, int kind, TcGroupInst &g)
{
    const int mt = t->pair ? 256 : TC_BM;
    if (kind == GP_TCG_ADJOINT) {
        g.A_hi = t->m_fxt_hi;
        g.A_lo = t->m_fxt_lo;
        g.A_x = t->m_fxt_hi;
        g.B_hi = t->m_w_hi;
        g.B_lo = t->m_w_lo;
        g.B_x = t->m_w_hi;
        g.m_tiles = t->xrows_pad / mt;
        g.n_tiles = t->M_pad / TC_BN;
        g.kb_total = t->K2_pad / t->bk;
        g.kb_per_split = t->kb_per;
        g.units = g.m_tiles * g.n_tiles * t->splits;
        g.gpart = c->gpart;
        g.out_ld = c->N;
        g.out_rows = c->N;
        g.out_cols = c->N;
        return;
    }
    const bool batch = kind == GP_TCG_TRIALS;
    const TcMaps fm = tc_fwd_maps(t, batch);
    g.A_hi = *fm.a_hi;
    g.A_lo = *fm.a_lo;
    g.A_x = *fm.a_x;
    g.B_hi = *fm.b_hi;
    g.B_lo = *fm.b_lo;
    g.B_x = *fm.b_x;
    g.m_tiles = t->rows_pad / mt;
    g.n_tiles = batch ? (GP_NTR * t->Lb) / TC_BN : t->M_pad / TC_BN;
    g.kb_total = t->Kx_pad / t->bk;
    g.kb_per_split = g.kb_total;
    g.units = g.m_tiles * g.n_tiles;
    g.fya = t->fya;
    g.fyr = t->fyr;
    g.nanc = t->nanc;
    g.nuv = c->nuv;
    if (batch) {
        g.lpad = t->Lb;
        const int erows = t->Lb < TC_EPI_COLS ? t->Lb : TC_EPI_COLS;
        g.elog2 = erows == 32 ? 5 : erows == 64 ? 6 : 7;
        g.rsc = t->rscb;
        g.vpart = c->vpart_b;
    } else {
        g.lpad = t->M_pad;  // one image, partial entries of TC_EPI_COLS rows
        g.elog2 = 7;
        g.rsc = t->rsc;
        g.vpart = c->vpart;
    }
}

// Builds the group of ctx[0..n-1] for a contraction of kind GP_TCG_* (their
// tensor state and batch buffers are allocated here if needed).
// GPAIR_ERR_STATE when the instances cannot share one launch (a CUDA-core
// instance, or another operand kind or tile layout).
int gp_tc_group_build_kind(gpair_ctx **ctx, int n, int kind, const int *gate, unsigned int *err, void **out)
{
    *out = nullptr;
    if (n <= 0 || n > TC_GROUP_MAX) return GPAIR_ERR_STATE;
    if (kind < GP_TCG_TRIALS || kind > GP_TCG_ADJOINT) return GPAIR_ERR_INVALID;
    TcGroupInst *h = (TcGroupInst *)calloc((size_t)n, sizeof(TcGroupInst));
    if (!h) return GPAIR_ERR_ALLOC;
    int rc = GPAIR_OK;
    TcState *t0 = nullptr;
    for (int i = 0; i < n && !rc; i++) {
        gpair_ctx *c = ctx[i];
        if (c->precision == GPAIR_PREC_FP32) {
            rc = GPAIR_ERR_STATE;
            break;
        }
        TcState *t = tc_state_ready(c, &rc);
        if (rc) break;
        if (kind == GP_TCG_TRIALS && (rc = gp_batch_alloc(c))) break;
        // the adjoint is the same contraction for both forward operand kinds of an op
        if (t0 && ((kind == GP_TCG_ADJOINT ? t->op != t0->op : t->fop != t0->fop) || t->nprod != t0->nprod ||
                   t->pair != t0->pair)) {
            rc = GPAIR_ERR_STATE;
            break;
        }
        if (!t0) t0 = t;
        tc_group_inst(c, t, kind, h[i]);
    }
    TcGroup *G = nullptr;
    if (!rc) {
        G = (TcGroup *)calloc(1, sizeof(TcGroup));
        if (!G) rc = GPAIR_ERR_ALLOC;
    }
    if (!rc) {
        G->n = n;
        G->epi = kind == GP_TCG_ADJOINT ? EPI_STORE : EPI_FWD;
        G->op = kind == GP_TCG_ADJOINT ? t0->op : t0->fop;
        G->nprod = t0->nprod;
        G->pair = t0->pair;
        G->npairs = t0->npairs;
        G->nsm = t0->nsm;
        G->map0 = h[0].A_hi;
        G->gate = gate;
        G->err = err;
        gpair_ctx *c = ctx[0];
        if (cudaMalloc(&G->d_inst, sizeof(TcGroupInst) * (size_t)n) != cudaSuccess ||
            cudaMemcpy(G->d_inst, h, sizeof(TcGroupInst) * (size_t)n, cudaMemcpyHostToDevice) != cudaSuccess) {
            snprintf(c->last_error, sizeof(c->last_error), "grouped contraction: device arrays");
            rc = GPAIR_ERR_CUDA;
        }
    }
    free(h);
    if (rc) {
        gp_tc_group_free(G);
        return rc;
    }
    *out = G;
    return GPAIR_OK;
}

int gp_tc_group_build(gpair_ctx **ctx, int n, const int *gate, unsigned int *err, void **out)
{
    return gp_tc_group_build_kind(ctx, n, GP_TCG_TRIALS, gate, err, out);
}

template <int EPI, int PAIR>
static cudaError_t tc_group_launch_kind(TcGroup *G, cudaStream_t st, int pdl, const TcArgs &a)
{
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cudaLaunchAttribute at[2];
    cfg.gridDim = dim3(PAIR ? 2 * (unsigned)G->npairs : (unsigned)G->nsm, 1, 1);
    cfg.blockDim = dim3(tc_threads<EPI>(), 1, 1);
    cfg.dynamicSmemBytes = TC_SMEM_GROUP_BYTES;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = tc_attrs(at, PAIR, pdl);
    const CUtensorMap &m = G->map0;
    if (EPI == EPI_FWD && G->op == OP_F16F8)
        return cudaLaunchKernelEx(&cfg, k_tc_gemm<EPI_FWD, OP_F16F8, 3, PAIR, 1>, m, m, m, m, m, m, a);
    if (G->op == OP_F16) return cudaLaunchKernelEx(&cfg, k_tc_gemm<EPI, OP_F16, 3, PAIR, 1>, m, m, m, m, m, m, a);
    if (G->nprod == 3) return cudaLaunchKernelEx(&cfg, k_tc_gemm<EPI, OP_TF32, 3, PAIR, 1>, m, m, m, m, m, m, a);
    return cudaLaunchKernelEx(&cfg, k_tc_gemm<EPI, OP_TF32, 1, PAIR, 1>, m, m, m, m, m, m, a);
}

// the grouped contraction of every gated instance, on stream st (persistent:
// one CTA per SM or one pair per two SMs, whatever the number of gated units);
// c gives the wait budget and the failure-test switch
int gp_tc_group_run(void *grp, gpair_ctx *c, cudaStream_t st)
{
    TcGroup *G = (TcGroup *)grp;
    TcArgs a;
    memset(&a, 0, sizeof(a));
    a.grp = G->d_inst;
    a.gate = G->gate;
    a.ninst = G->n;
    a.err = G->err;
    a.budget = c->tc_wait_budget > 0 ? c->tc_wait_budget : TC_WAIT_BUDGET;
    a.skip_loads = c->tc_skip_loads;
    cudaError_t e;
    if (G->epi == EPI_STORE)
        e = G->pair ? tc_group_launch_kind<EPI_STORE, 1>(G, st, c->pdl, a)
                    : tc_group_launch_kind<EPI_STORE, 0>(G, st, c->pdl, a);
    else
        e = G->pair ? tc_group_launch_kind<EPI_FWD, 1>(G, st, c->pdl, a)
                    : tc_group_launch_kind<EPI_FWD, 0>(G, st, c->pdl, a);
    if (e != cudaSuccess) {
        snprintf(c->last_error, sizeof(c->last_error), "grouped contraction launch: %s", cudaGetErrorString(e));
        return GPAIR_ERR_CUDA;
    }
    c->launches++;
    return GPAIR_OK;
}

int gp_tc_group_forward(void *grp, gpair_ctx *c) { return gp_tc_group_run(grp, c, c->stream); }

// ------------------------------------------------- grouped stage launches
//
// The tensor path's own stages of a lockstep iteration as one launch over all
// instances (group.cuh): the current image's prep (flux, regulariser, max and
// forward operand), the batched trials' prep, and the adjoint weight operand.

// partial visibility entries of the forward of one N x N image (rows of TC_EPI_COLS)
int gp_tc_forward_entries(int N) { return round_up(N, TC_BN) / TC_EPI_COLS; }

int gp_tc_stage_sizes(gpair_ctx *c, int *mt, int *splits)
{
    int rc;
    TcState *t = tc_state_ready(c, &rc);
    if (rc) return rc;
    if (mt) *mt = t->M_pad / TC_EPI_COLS;
    if (splits) *splits = t->splits;
    return GPAIR_OK;
}

size_t gp_tc_stage_args_size(int stage)
{
    switch (stage) {
    case GS_PREP_IMAGE:
    case GS_PREP_TRIALS: return sizeof(PrepRowsArgs);
    case GS_BUILD_W: return sizeof(BuildWArgs);
    default: return 0;
    }
}

// blocks of one trial image in the trial prep when a block takes `passes`
// passes of rows (per-row sums, rows one warp wide) or the single launch's grid
static int tc_prep_trial_blocks(int N, int passes)
{
    const int W = pr_warps_per_row(N), R = PR_WARPS_MAX / W;
    int gx = gp_cdiv(N, R);
    if (gx > 1024) gx = 1024;
    if (W == 1 && passes > 1) gx = gp_cdiv(gx, passes);
    return gx < 1 ? 1 : gx;
}

int gp_tc_stage_args(gpair_ctx *c, int stage, void *out, int *nblocks, int *op, int passes)
{
    int rc;
    TcState *t = tc_state_ready(c, &rc);
    if (rc) return rc;
    *op = t->op;
    if (stage == GS_PREP_IMAGE || stage == GS_PREP_TRIALS) {
        if (stage == GS_PREP_TRIALS && (rc = gp_tc_batch_prepare(c, nullptr))) return rc;
        PrepRowsArgs a = stage == GS_PREP_IMAGE ? tc_prep_rows_args(c, t, 0, 1, c->partials, c->image)
                                                : tc_prep_rows_args(c, t, 2, 1, c->partials_b, nullptr);
        if (stage == GS_PREP_TRIALS) a.nbx = tc_prep_trial_blocks(c->N, passes);
        memcpy(out, &a, sizeof(a));
        *nblocks = a.nbx * a.nby;
        return GPAIR_OK;
    }
    if (stage == GS_BUILD_W) {
        if (!c->have_uv) return GPAIR_ERR_STATE;  // the table-only path reads Fy from its table
        const BuildWArgs a = tc_build_w_args(c, t);
        memcpy(out, &a, sizeof(a));
        *nblocks = a.nbx * a.nby;
        return GPAIR_OK;
    }
    return GPAIR_ERR_INVALID;
}

// Passes of rows per block for the grouped trial prep of a staged batch: the
// smallest power of two that brings the launch (every instance's 8 trial
// images) within four waves of resident blocks. One pass per block leaves the
// launch bound by each block's fixed start and end (instance lookup, scalars,
// the last-block reduction): 80 registers a thread give 3 blocks of 256 per SM.
int gp_tc_prep_trials_passes(gpair_ctx *const *ctx, int n, int op)
{
    if (n < 1) return 1;
    int nsm = 0, per = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx[0]->device) != cudaSuccess || nsm < 1)
        return 1;
    const cudaError_t e =
        op == OP_F16
            ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_grouped<PrepRowsOp<__half, 2>, PR_THREADS>,
                                                            PR_THREADS, 0)
            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_grouped<PrepRowsOp<float, 2>, PR_THREADS>,
                                                            PR_THREADS, 0);
    if (e != cudaSuccess || per < 1) return 1;
    const long long waves4 = 4LL * per * nsm;
    int p = 1;
    for (; p < 32; p *= 2) {
        long long total = 0;
        for (int k = 0; k < n; k++) total += (long long)GP_NTR * tc_prep_trial_blocks(ctx[k]->N, p);
        if (total <= waves4) break;
    }
    return p;
}

template <class Op, int THREADS>
static int tc_group_stage(gpair_ctx *c, const void *d_args, const int *d_start, int n, int total, const int *gate)
{
    GP_LAUNCH(c, gp_launch(c, k_grouped<Op, THREADS>, dim3(total), dim3(THREADS), 0,
                           (const typename Op::Args *)d_args, d_start, n, gate));
    return GPAIR_OK;
}

int gp_tc_stage_group_launch(gpair_ctx *c, int stage, int op, const void *d_args, const int *d_start, int n,
                             int total, const int *gate)
{
    if (total < 1 || n < 1) return GPAIR_ERR_INVALID;
    const bool f16 = op == OP_F16;
    switch (stage) {
    case GS_PREP_IMAGE:
        return f16 ? tc_group_stage<PrepRowsOp<__half, 0>, PR_THREADS>(c, d_args, d_start, n, total, gate)
                   : tc_group_stage<PrepRowsOp<float, 0>, PR_THREADS>(c, d_args, d_start, n, total, gate);
    case GS_PREP_TRIALS:
        return f16 ? tc_group_stage<PrepRowsOp<__half, 2>, PR_THREADS>(c, d_args, d_start, n, total, gate)
                   : tc_group_stage<PrepRowsOp<float, 2>, PR_THREADS>(c, d_args, d_start, n, total, gate);
    case GS_BUILD_W:
        return f16 ? tc_group_stage<BuildWOp<__half>, 256>(c, d_args, d_start, n, total, gate)
                   : tc_group_stage<BuildWOp<float>, 256>(c, d_args, d_start, n, total, gate);
    default: return GPAIR_ERR_INVALID;
    }
}
