// Learned Spalart-Allmaras source: an MLP 6 -> 64 -> 64 -> 64 -> 1 (SiLU) that
// replaces production - wall destruction of SourceFluxOneEquationOriginal
// (CFD/TurbSolver/src/TurbSolverUnstr.cpp:2702-2916) inside its training hull;
// the exact source is used outside it and for nu~ <= 0.
//
// Inference runs on the 5th-generation tensor cores: per CTA a tile of 128
// cells, FP16 operands in shared memory (canonical K-major layout, no
// swizzle), FP32 accumulators in tensor memory (TMEM), tcgen05.mma issued by
// one thread and completed through an mbarrier, results read back with
// tcgen05.ld.  The last layer (64 -> 1) is a dot product on the CUDA cores.
// Training uses hand-written FP32 forward / backward / Adam kernels.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "phx_device.cuh"
#include "phx_internal.h"
#include "phx_mlp.h"
#include "phx_sa.cuh"

namespace phx {

// ---------------------------------------------------------------------------
// tcgen05 / TMEM / mbarrier helpers (inline PTX, sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: canonical K-major layout without swizzle,
// core matrices of 8 rows x 16 bytes; lbo = byte distance between the two
// 8-element K chunks of one MMA, sbo = byte distance between 8-row groups;
// version 1 (sm_100) in bits 46-47, layout type 0 (no swizzle) in bits 61-63.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16: D FP32 (bits 4-5 = 1), A and B FP16
// (bits 7-9 = 0, 10-12 = 0), both K-major, N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t umma_idesc_f16(int M, int N)
{
    return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

// Bounded wait for the mbarrier phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity)
{
    const uint32_t a = smem_u32(mbar);
    for (long long i = 0; i < (1LL << 26); ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 lanes x 64 columns of FP32 from TMEM into 64 registers per thread.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float *v)
{
    uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
        "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
        "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

// SiLU of a pair, x sigma(x) = x/2 + (x/2) tanh(x/2), with one
// tanh.approx.f16x2 for both values: one special-function operation per two
// activations instead of an exponential and a reciprocal per activation.  The
// last hidden layer uses it in FP32 (its outputs go to the CUDA-core dot
// product); the half-precision tanh of x/2 has a relative error of ~2^-11.
__device__ __forceinline__ void silu2(float &a, float &b)
{
    const float ha = 0.5f * a, hb = 0.5f * b;
    const __half2 h = __floats2half2_rn(ha, hb);
    uint32_t t;
    asm("tanh.approx.f16x2 %0, %1;" : "=r"(t) : "r"(*reinterpret_cast<const uint32_t *>(&h)));
    const float2 tf = __half22float2(*reinterpret_cast<const __half2 *>(&t));
    a = fmaf(ha, tf.x, ha);
    b = fmaf(hb, tf.y, hb);
}

// ---------------------------------------------------------------------------
// Features and target of the learned source, for a cell with nu~ > 0.
// rate = nu~ / (d^2 Re) is the destruction rate scale.  With ft2 = 0 the
// NSMB source (TurbSolverUnstr.cpp:2790-2870) divided by nu~ rate is a
// function of two variables only, chi = nu~ rho / mu and s = Omega / rate:
// S~ / rate = s + fv2(chi) / kappa^2 (or its clipped form), r = 1 / (kappa^2
// S~ / rate), src / (nu~ rate) = cb1 S~ / rate - cw1 fw(r).  The target
// t = src / (nu~ rate (1 + s)) stays of order one, and the six inputs are
// smooth functions of (chi, s), so the model learns that two-variable
// function and nothing that varies between states or precisions at equal
// (chi, s):
//   f0 = ln chi, f1 = ln s, f2 = fv1(chi), f3 = s / (1 + s), f4 = 1 / (1 + chi),
//   f5 = ln(1 + s).
// s is floored at kRateFloor: below it the source is within 0.1 % of its
// s = 0 value (S~ is clipped and r = 10 when fv2 < 0; S~ / rate moves by
// 1e-3 otherwise), and a near-uniform region, where the velocity gradients of
// an FP32 state are exactly zero and those of an FP64 state are round-off,
// maps to one finite point in both precisions.
// ---------------------------------------------------------------------------
constexpr float kRateFloor = 1e-3f;

__device__ __forceinline__ void sa_features(float nue, float omega, float olam, float d, float oRe, float *f,
                                            float &scale)
{
    const float rate = nue * oRe / (d * d);
    const float chi = nue * olam;
    const float sr = omega / rate;
    const float s = fmaxf(sr, kRateFloor);
    const float chi3 = chi * chi * chi;
    f[0] = __logf(chi);
    f[1] = __logf(s);
    f[2] = chi3 / (chi3 + 357.911f);   // fv1, cv1 = 7.1
    f[3] = s / (1.0f + s);
    f[4] = 1.0f / (1.0f + chi);
    f[5] = log1pf(s);
    scale = nue * rate * (1.0f + sr);
}

// Inputs of the source for one cell: vorticity magnitude of the NS velocity
// gradients, nu~, rho / mu, wall distance.
template <class T>
__device__ __forceinline__ void sa_cell_inputs(const DevGrid &g, const Work<T> &w, int cell, T &nue, T &omega,
                                               T &olam, double &d)
{
    T tr[4];
    ld4(w.trec + (size_t)cell * kTr, tr);
    nue = tr[0];
    const T rho = w.qrec[(size_t)cell * kQ];
    T gr[16];
    const T *gp = w.grec + (size_t)cell * kG;
    ld8(gp, gr);
    ld8(gp + 8, gr + 8);
    const T dudy = gr[4], dudz = gr[5], dvdx = gr[6], dvdz = gr[8], dwdx = gr[9], dwdy = gr[10];
    omega = sqrt((dwdy - dvdz) * (dwdy - dvdz) + (dudz - dwdx) * (dudz - dwdx) + (dvdx - dudy) * (dvdx - dudy));
    olam = rho / (tr[2] + (T)kSmall);
    d = ld(g.walldist + cell);
}

// ---------------------------------------------------------------------------
// Inference: source of every cell into t.tsrc (the SA cell pass reads it).
// One CTA = 128 threads = one row of the 128-cell tile each; persistent over
// tiles.  Shared memory: W1 | W2 | W3 | A1 (128 x 16) | ACT (128 x 64) | b1, b2
// in half precision | mbarrier, TMEM address.  Operands are FP16: the input
// row, the weights, and the hidden activations, which the half-precision
// epilogue writes as they are.
// ---------------------------------------------------------------------------
static constexpr int kMlpSmemW1 = 0;
static constexpr int kMlpSmemW2 = kMlpSmemW1 + kMlpH * kMlpK1 * 2;
static constexpr int kMlpSmemW3 = kMlpSmemW2 + kMlpH * kMlpH * 2;
static constexpr int kMlpSmemA1 = kMlpSmemW3 + kMlpH * kMlpH * 2;
static constexpr int kMlpSmemAct = kMlpSmemA1 + kMlpTile * kMlpK1 * 2;
static constexpr int kMlpSmemBias = kMlpSmemAct + kMlpTile * kMlpH * 2;   // b1, b2 as half2 pairs
static constexpr int kMlpSmemBar = kMlpSmemBias + 2 * kMlpH * 2;
static constexpr int kMlpSmemBytes = kMlpSmemBar + 16;
static constexpr uint32_t kMlpTmemCols = 64;

// Row r of a K-major FP16 tile with `kchunks` 8-element K chunks (sbo = kchunks * 128),
// from FP32 values or from packed pairs.
__device__ __forceinline__ void store_row_f16(unsigned char *base, int r, int kchunks, const float *v)
{
    unsigned char *row = base + (r >> 3) * (kchunks * 128) + (r & 7) * 16;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        if (c >= kchunks) break;
        __half2 p[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) p[i] = __floats2half2_rn(v[8 * c + 2 * i], v[8 * c + 2 * i + 1]);
        *reinterpret_cast<uint4 *>(row + c * 128) = *reinterpret_cast<uint4 *>(p);
    }
}
__device__ __forceinline__ void store_row_h2(unsigned char *base, int r, const __half2 *v)
{
    unsigned char *row = base + (r >> 3) * ((kMlpH / 8) * 128) + (r & 7) * 16;
#pragma unroll
    for (int c = 0; c < kMlpH / 8; ++c) *reinterpret_cast<uint4 *>(row + c * 128) = *reinterpret_cast<const uint4 *>(v + 4 * c);
}

// Bias and SiLU of a hidden layer whose output feeds the next MMA, in half
// precision: per pair of FP32 accumulators one pack, then the bias, x/2,
// tanh(x/2) (one tanh.approx.f16x2) and x/2 + (x/2) tanh(x/2) in half2
// arithmetic, so the result is the next layer's FP16 operand as it stands.
__device__ __forceinline__ void bias_silu_h2(const float *acc, const __half2 *bias2, __half2 *out)
{
    const __half2 half = __float2half2_rn(0.5f);
#pragma unroll
    for (int k = 0; k < kMlpH / 2; ++k) {
        const __half2 x = __hadd2(__floats2half2_rn(acc[2 * k], acc[2 * k + 1]), bias2[k]);
        const __half2 hx = __hmul2(x, half);
        uint32_t t;
        asm("tanh.approx.f16x2 %0, %1;" : "=r"(t) : "r"(*reinterpret_cast<const uint32_t *>(&hx)));
        out[k] = __hfma2(hx, *reinterpret_cast<const __half2 *>(&t), hx);
    }
}

template <class T>
__global__ void __launch_bounds__(kMlpTile, 5) mlp_source_kernel(DevGrid g, NsConst c, Work<T> w, TurbWork<T> t,
                                                               MlpDev mlp, Reduce *red, unsigned long long *nmlp)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + kMlpSmemBar);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + kMlpSmemBar + 8);
    const int tid = threadIdx.x, warp = tid >> 5;
    // weights to shared memory (already in the MMA layout)
    {
        const uint4 *s1 = reinterpret_cast<const uint4 *>(mlp.w1c);
        const uint4 *s2 = reinterpret_cast<const uint4 *>(mlp.w2c);
        const uint4 *s3 = reinterpret_cast<const uint4 *>(mlp.w3c);
        uint4 *d1 = reinterpret_cast<uint4 *>(sm + kMlpSmemW1);
        uint4 *d2 = reinterpret_cast<uint4 *>(sm + kMlpSmemW2);
        uint4 *d3 = reinterpret_cast<uint4 *>(sm + kMlpSmemW3);
        for (int i = tid; i < kMlpH * kMlpK1 * 2 / 16; i += blockDim.x) d1[i] = s1[i];
        for (int i = tid; i < kMlpH * kMlpH * 2 / 16; i += blockDim.x) { d2[i] = s2[i]; d3[i] = s3[i]; }
        __half2 *bh = reinterpret_cast<__half2 *>(sm + kMlpSmemBias);
        if (tid < kMlpH) {
            const float *b = tid < kMlpH / 2 ? mlp.b1 : mlp.b2;
            const int k = 2 * (tid % (kMlpH / 2));
            bh[tid] = __floats2half2_rn(__ldg(b + k), __ldg(b + k + 1));
        }
    }
    if (tid == 0) {
        mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kMlpTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);   // this warp's 32 lanes
    const uint32_t idesc = umma_idesc_f16(kMlpTile, kMlpH);
    const uint32_t sW1 = smem_u32(sm + kMlpSmemW1), sW2 = smem_u32(sm + kMlpSmemW2), sW3 = smem_u32(sm + kMlpSmemW3);
    const uint32_t sA1 = smem_u32(sm + kMlpSmemA1), sAct = smem_u32(sm + kMlpSmemAct);
    uint32_t phase = 0;
    bool ok = true;
    unsigned long long used = 0;
    const int ntiles = (g.nCell + kMlpTile - 1) / kMlpTile;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int cell = tile * kMlpTile + tid;
        // inputs and features (the exact source of fallback cells is formed by the SA cell pass)
        float x[kMlpK1];
#pragma unroll
        for (int k = 0; k < kMlpK1; ++k) x[k] = 0.0f;
        float scale = 0.0f;
        bool useMlp = false;
        if (cell < g.nCell) {
            T nue, omega, olam;
            double d;
            sa_cell_inputs<T>(g, w, cell, nue, omega, olam, d);
            if (nue > T(0) && c.saSource) {
                float f[kMlpIn];
                sa_features((float)nue, (float)omega, (float)olam, (float)d, (float)c.oRe, f, scale);
                useMlp = true;
#pragma unroll
                for (int k = 0; k < kMlpIn; ++k) {
                    if (c.saSource == 2 && !(f[k] >= mlp.lo[k] && f[k] <= mlp.hi[k])) useMlp = false;
                    x[k] = (f[k] - mlp.mean[k]) * mlp.rstd[k];
                }
                // inside the box, the (chi, s) bin must hold training samples
                if (c.saSource == 2 && useMlp)
                    useMlp = __ldg(mlp.occ + mlp_bin(f[0], mlp.lo[0], mlp.hi[0]) * kMlpGrid +
                                   mlp_bin(f[1], mlp.lo[1], mlp.hi[1])) != 0;
            }
        }
        // the next tile's cell records into L2 while this tile's MMAs run
        {
            const int nxt = cell + gridDim.x * kMlpTile;
            if (nxt < g.nCell) {
                prefetch_l2(w.grec + (size_t)nxt * kG);
                prefetch_l2(w.grec + (size_t)nxt * kG + 8);
                prefetch_l2(w.trec + (size_t)nxt * kTr);
                prefetch_l2(w.qrec + (size_t)nxt * kQ);
                prefetch_l2(g.walldist + nxt);
            }
        }
        store_row_f16(sm + kMlpSmemA1, tid, kMlpK1 / 8, x);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // layer 1: [128 x 16] x [16 x 64]
        if (tid == 0) {
            umma_f16(tmem, umma_desc(sA1, 128, 256), umma_desc(sW1, 128, 256), idesc, 0u);
            umma_commit(mbar);
        }
        float h[kMlpH];
#pragma unroll
        for (int layer = 0; layer < 3; ++layer) {
            // every thread leaves together if the MMA did not complete in time
            if (!__syncthreads_and(mbar_wait(mbar, phase) ? 1 : 0)) { ok = false; break; }
            phase ^= 1u;
            tc_fence_after();
            tmem_ld64(taddr, h);
            if (layer == 2) {
                // the last hidden layer feeds the CUDA-core dot product: FP32
#pragma unroll
                for (int k = 0; k < kMlpH; k += 2) {
                    h[k] += __ldg(mlp.b3 + k);
                    h[k + 1] += __ldg(mlp.b3 + k + 1);
                    silu2(h[k], h[k + 1]);
                }
                break;
            }
            __half2 a2[kMlpH / 2];
            bias_silu_h2(h, reinterpret_cast<const __half2 *>(sm + kMlpSmemBias) + layer * (kMlpH / 2), a2);
            store_row_h2(sm + kMlpSmemAct, tid, a2);
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            if (tid == 0) {
                const uint32_t sW = layer == 0 ? sW2 : sW3;
#pragma unroll
                for (int kk = 0; kk < kMlpH / 16; ++kk)
                    umma_f16(tmem, umma_desc(sAct + kk * 256, 128, 1024), umma_desc(sW + kk * 256, 128, 1024), idesc,
                              kk > 0 ? 1u : 0u);
                umma_commit(mbar);
            }
        }
        if (!ok) break;
        // layer 4 on the CUDA cores
        float out = mlp.b4;
#pragma unroll
        for (int k = 0; k < kMlpH; ++k) out += __ldg(mlp.w4 + k) * h[k];
        if (cell < g.nCell) {
            // NaN marks a cell that takes the exact source
            t.tsrc[cell] = useMlp ? (T)(out * mlp.tscale * scale) : (T)__int_as_float(0x7fc00000);
            used += useMlp ? 1 : 0;
        }
        tc_fence_before();
        __syncthreads();   // TMEM reads of this tile done before the next tile's MMA
        tc_fence_after();
    }
    if (!ok && tid == 0) atomicExch(&red->error, PHX_ERR_TIMEOUT);
    for (int o = 16; o > 0; o >>= 1) used += __shfl_xor_sync(0xffffffffu, used, o);
    if ((tid & 31) == 0 && used) atomicAdd(nmlp, used);
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMlpTmemCols));
}

template <class T>
void launch_mlp_source(const DevGrid &g, const NsConst &c, const Work<T> &w, const TurbWork<T> &t,
                       const MlpDev &mlp, Reduce *red, unsigned long long *nmlp, int numSMs, cudaStream_t s)
{
    // the attribute is per device: set on the current one at every launch
    // (microseconds)
    cudaFuncSetAttribute(mlp_source_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMlpSmemBytes);
    const int ntiles = (g.nCell + kMlpTile - 1) / kMlpTile;
    // persistent CTAs, every one resident: 5 per SM use 5 x 64 of the 512 TMEM
    // columns, 5 x 39 KB shared memory and 5 x 128 threads x at most 102
    // registers (the kernel's launch bounds)
    int blocks = numSMs * 5;
    if (blocks > ntiles) blocks = ntiles;
    if (blocks < 1) blocks = 1;
    mlp_source_kernel<T><<<blocks, kMlpTile, kMlpSmemBytes, s>>>(g, c, w, t, mlp, red, nmlp);
}

// Training samples of every cell with nu~ > 0: raw features and the target
// t = src / scale of the exact source (written compactly through an atomic slot).
template <class T>
__global__ void __launch_bounds__(kThreads) mlp_capture_kernel(DevGrid g, NsConst c, Work<T> w, TurbWork<T> t,
                                                                float *feat, float *targ, int *cells, float *scales,
                                                                long long cap, unsigned long long *count)
{
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.nCell) return;
    T nue, omega, olam;
    double d;
    sa_cell_inputs<T>(g, w, cell, nue, omega, olam, d);
    if (!(nue > T(0))) return;
    T src, sspec;
    sa_source_fp64<T>(nue, omega, olam, d, T(0), c.oRe, src, sspec);
    float f[kMlpIn], scale;
    sa_features((float)nue, (float)omega, (float)olam, (float)d, (float)c.oRe, f, scale);
    const unsigned long long slot = atomicAdd(count, 1ULL);
    if ((long long)slot >= cap) return;
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) feat[slot * kMlpIn + k] = f[k];
    targ[slot] = (float)src / scale;
    cells[slot] = g.orig[cell];
    scales[slot] = scale;
}

template <class T>
void launch_mlp_capture(const DevGrid &g, const NsConst &c, const Work<T> &w, const TurbWork<T> &t, float *feat,
                        float *targ, int *cells, float *scales, long long cap, unsigned long long *count,
                        cudaStream_t s)
{
    mlp_capture_kernel<T><<<(g.nCell + kThreads - 1) / kThreads, kThreads, 0, s>>>(g, c, w, t, feat, targ, cells,
                                                                                  scales, cap, count);
}

// ---------------------------------------------------------------------------
// Training (FP32, CUDA cores): C[M x N] (+)= op(A) op(B) with element strides
// A(i, k) = A[i * as0 + k * as1], B(k, j) = B[k * bs0 + j * bs1]; 16 x 16 tiles.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) mlp_gemm_kernel(int M, int N, int K, const float *A, long long as0,
                                                       long long as1, const float *B, long long bs0, long long bs1,
                                                       float *C, int ldc, const float *bias, int accumulate)
{
    __shared__ float sa[16][17], sb[16][17];
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
    const int i = blockIdx.y * 16 + ty, j = blockIdx.x * 16 + tx;
    float acc = 0.0f;
    for (int k0 = 0; k0 < K; k0 += 16) {
        const int ka = k0 + tx, kb = k0 + ty;
        sa[ty][tx] = (i < M && ka < K) ? A[i * as0 + ka * as1] : 0.0f;
        sb[ty][tx] = (kb < K && j < N) ? B[kb * bs0 + j * bs1] : 0.0f;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) acc += sa[ty][k] * sb[k][tx];
        __syncthreads();
    }
    if (i < M && j < N) {
        if (bias) acc += bias[j];
        float *cp = C + (size_t)i * ldc + j;
        *cp = accumulate ? *cp + acc : acc;
    }
}

void mlp_gemm(int M, int N, int K, const float *A, long long as0, long long as1, const float *B, long long bs0,
              long long bs1, float *C, int ldc, const float *bias, bool accumulate, cudaStream_t s)
{
    dim3 grid((N + 15) / 16, (M + 15) / 16);
    mlp_gemm_kernel<<<grid, 256, 0, s>>>(M, N, K, A, as0, as1, B, bs0, bs1, C, ldc, bias, accumulate ? 1 : 0);
}

// h = silu(z) (forward) or dz = dh * silu'(z) (backward), n elements.
__global__ void mlp_silu_kernel(long long n, const float *z, float *h, const float *dh, float *dz)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x = z[i];
    const float sg = 1.0f / (1.0f + expf(-x));
    if (h) h[i] = x * sg;
    if (dz) dz[i] = dh[i] * (sg * (1.0f + x * (1.0f - sg)));
}

void mlp_silu(long long n, const float *z, float *h, const float *dh, float *dz, cudaStream_t s)
{
    mlp_silu_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, z, h, dh, dz);
}

// Rows gathered from the sample set by a permutation: x[b] = X[perm[off + b]].
__global__ void mlp_gather_kernel(int nb, const int *perm, int off, const float *X, const float *Y, float *x, float *y,
                                  const float *mean, const float *rstd, float tinv)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const int r = perm[off + b];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) x[b * kMlpIn + k] = (X[(size_t)r * kMlpIn + k] - mean[k]) * rstd[k];
    y[b] = Y[r] * tinv;
}

// dy = 2 (y - t) / nb, and the squared error summed per block into loss[blockIdx.x]
// (fixed order: warp shuffles, then the block's warps in order; the host sums
// the block partials in order, so the reported loss does not depend on timing).
__global__ void __launch_bounds__(256) mlp_loss_kernel(int nb, const float *y, const float *t, float *dy, float *loss)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    float e = 0.0f;
    if (b < nb) {
        const float r = y[b] - t[b];
        dy[b] = 2.0f * r / nb;
        e = r * r;
    }
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    __shared__ float part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        float acc = 0.0f;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) acc += part[i];
        loss[blockIdx.x] += acc;
    }
}

// Column sums of a [rows x cols] matrix (bias gradients).
__global__ void mlp_colsum_kernel(int rows, int cols, const float *a, float *out)
{
    const int j = blockIdx.x;
    float s = 0.0f;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) s += a[(size_t)i * cols + j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ float part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += part[i];
        out[j] = t;
    }
}

// Adam (Kingma & Ba 2015) over the flat parameter vector.
__global__ void mlp_adam_kernel(int n, float *p, const float *gr, float *m, float *v, float lr, float b1, float b2,
                                float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = gr[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

void mlp_train_kernels_launch_silu_cols(int rows, int cols, const float *a, float *out, cudaStream_t s)
{
    mlp_colsum_kernel<<<cols, 256, 0, s>>>(rows, cols, a, out);
}

// ---------------------------------------------------------------------------
// Host side: training driver and packing of the weights into the MMA layout.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNW1 = kMlpH * kMlpIn, kNW2 = kMlpH * kMlpH, kNW3 = kMlpH * kMlpH;
// flat parameter vector: w1 b1 w2 b2 w3 b3 w4 b4
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kNW1, kOffW2 = kOffB1 + kMlpH, kOffB2 = kOffW2 + kNW2;
constexpr int kOffW3 = kOffB2 + kMlpH, kOffB3 = kOffW3 + kNW3, kOffW4 = kOffB3 + kMlpH, kOffB4 = kOffW4 + kMlpH;
constexpr int kNParam = kOffB4 + 1;

struct DevBuf {
    std::vector<void *> p;
    ~DevBuf() { for (void *q : p) cudaFree(q); }
    template <class T> T *get(size_t n)
    {
        void *v = nullptr;
        if (cudaMalloc(&v, n * sizeof(T) > 0 ? n * sizeof(T) : 1) != cudaSuccess) return nullptr;
        p.push_back(v);
        return static_cast<T *>(v);
    }
};

// splitmix64 (Steele, Lea & Flood 2014) for the seeded initialisation and shuffles
uint64_t splitmix(uint64_t &x)
{
    uint64_t z = (x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
float uniform(uint64_t &x) { return (float)((splitmix(x) >> 11) * (1.0 / 9007199254740992.0)); }

}  // namespace

// Flat parameter vector (w1 b1 w2 b2 w3 b3 w4 b4) and the activation buffers
// of one batch of B rows.
struct MlpBatch {
    float *z1, *h1, *z2, *h2, *z3, *h3, *dh, *dz, *yp, *dy;
};

// Forward pass of one batch (x: standardised inputs [B][6], yt: scaled
// targets [B]) and the gradient of the mean squared error into gp; the batch's
// squared error is added to loss[0 .. ceil(B / 256)).
void mlp_forward_backward(const float *p, float *gp, const float *x, const float *yt, int B, const MlpBatch &a,
                          float *loss, cudaStream_t s)
{
    const int H = kMlpH;
    // forward: z = a W^T + b (W row-major [out][in])
    mlp_gemm(B, H, kMlpIn, x, kMlpIn, 1, p + kOffW1, 1, kMlpIn, a.z1, H, p + kOffB1, false, s);
    mlp_silu((long long)B * H, a.z1, a.h1, nullptr, nullptr, s);
    mlp_gemm(B, H, H, a.h1, H, 1, p + kOffW2, 1, H, a.z2, H, p + kOffB2, false, s);
    mlp_silu((long long)B * H, a.z2, a.h2, nullptr, nullptr, s);
    mlp_gemm(B, H, H, a.h2, H, 1, p + kOffW3, 1, H, a.z3, H, p + kOffB3, false, s);
    mlp_silu((long long)B * H, a.z3, a.h3, nullptr, nullptr, s);
    mlp_gemm(B, 1, H, a.h3, H, 1, p + kOffW4, 1, 1, a.yp, 1, p + kOffB4, false, s);
    mlp_loss_kernel<<<(B + 255) / 256, 256, 0, s>>>(B, a.yp, yt, a.dy, loss);
    // backward
    mlp_gemm(1, H, B, a.dy, 1, 1, a.h3, H, 1, gp + kOffW4, H, nullptr, false, s);             // dW4 = dy^T h3
    mlp_train_kernels_launch_silu_cols(B, 1, a.dy, gp + kOffB4, s);                           // db4
    mlp_gemm(B, H, 1, a.dy, 1, 1, p + kOffW4, 1, 1, a.dh, H, nullptr, false, s);              // dH3 = dy w4
    mlp_silu((long long)B * H, a.z3, nullptr, a.dh, a.dz, s);                                 // dZ3
    mlp_gemm(H, H, B, a.dz, 1, H, a.h2, H, 1, gp + kOffW3, H, nullptr, false, s);             // dW3 = dZ3^T H2
    mlp_train_kernels_launch_silu_cols(B, H, a.dz, gp + kOffB3, s);
    mlp_gemm(B, H, H, a.dz, H, 1, p + kOffW3, H, 1, a.dh, H, nullptr, false, s);              // dH2 = dZ3 W3
    mlp_silu((long long)B * H, a.z2, nullptr, a.dh, a.dz, s);
    mlp_gemm(H, H, B, a.dz, 1, H, a.h1, H, 1, gp + kOffW2, H, nullptr, false, s);             // dW2
    mlp_train_kernels_launch_silu_cols(B, H, a.dz, gp + kOffB2, s);
    mlp_gemm(B, H, H, a.dz, H, 1, p + kOffW2, H, 1, a.dh, H, nullptr, false, s);              // dH1 = dZ2 W2
    mlp_silu((long long)B * H, a.z1, nullptr, a.dh, a.dz, s);
    mlp_gemm(H, kMlpIn, B, a.dz, 1, H, x, kMlpIn, 1, gp + kOffW1, kMlpIn, nullptr, false, s);  // dW1
    mlp_train_kernels_launch_silu_cols(B, H, a.dz, gp + kOffB1, s);
}

// Device buffers of one batch of B rows (nullptr members if an allocation failed).
static bool mlp_batch_alloc(DevBuf &db, int B, MlpBatch &a)
{
    const size_t bh = (size_t)B * kMlpH;
    a.z1 = db.get<float>(bh); a.h1 = db.get<float>(bh); a.z2 = db.get<float>(bh); a.h2 = db.get<float>(bh);
    a.z3 = db.get<float>(bh); a.h3 = db.get<float>(bh); a.dh = db.get<float>(bh); a.dz = db.get<float>(bh);
    a.yp = db.get<float>(B); a.dy = db.get<float>(B);
    return a.z1 && a.h1 && a.z2 && a.h2 && a.z3 && a.h3 && a.dh && a.dz && a.yp && a.dy;
}

// Trains the MLP on n samples (raw features [n][6], targets [n]) with Adam and
// mean-squared error; returns the weights, the normalisation, the hull (box
// and occupied bins), and the loss of the last epoch (normalised units).  0 on success, else a CUDA error.
int mlp_train(const float *X, const float *Y, long long n, int epochs, int batch, float lr, unsigned long long seed,
              MlpHostWeights &wts, float *mean, float *rstd, float *lo, float *hi, float *occ, float &tscale,
              double &lastLoss, cudaStream_t s)
{
    if (n < 2 || batch < 1) return -1;
    // normalisation and hull
    double sum[kMlpIn] = {0}, sq[kMlpIn] = {0}, ys = 0.0, yq = 0.0;
    for (int k = 0; k < kMlpIn; ++k) { lo[k] = 3.0e38f; hi[k] = -3.0e38f; }
    for (long long i = 0; i < n; ++i) {
        for (int k = 0; k < kMlpIn; ++k) {
            const double v = X[i * kMlpIn + k];
            sum[k] += v; sq[k] += v * v;
            lo[k] = std::min(lo[k], (float)v); hi[k] = std::max(hi[k], (float)v);
        }
        ys += Y[i]; yq += (double)Y[i] * Y[i];
    }
    for (int k = 0; k < kMlpIn; ++k) {
        mean[k] = (float)(sum[k] / n);
        const double var = std::max(sq[k] / n - (sum[k] / n) * (sum[k] / n), 1e-12);
        rstd[k] = (float)(1.0 / std::sqrt(var));
    }
    tscale = (float)std::sqrt(std::max(yq / n, 1e-30));
    // occupied (ln chi, ln s) bins: the learned source is used only where training samples fell
    for (int b = 0; b < kMlpGrid * kMlpGrid; ++b) occ[b] = 0.0f;
    for (long long i = 0; i < n; ++i)
        occ[mlp_bin(X[i * kMlpIn], lo[0], hi[0]) * kMlpGrid + mlp_bin(X[i * kMlpIn + 1], lo[1], hi[1])] = 1.0f;
    // initialisation (uniform, fan-in scaled)
    std::vector<float> prm(kNParam, 0.0f);
    uint64_t rs = seed * 0x2545F4914F6CDD1DULL + 1;
    auto init = [&](int off, int fanin, int count) {
        const float a = std::sqrt(3.0f / fanin);
        for (int i = 0; i < count; ++i) prm[off + i] = (2.0f * uniform(rs) - 1.0f) * a;
    };
    init(kOffW1, kMlpIn, kNW1);
    init(kOffW2, kMlpH, kNW2);
    init(kOffW3, kMlpH, kNW3);
    init(kOffW4, kMlpH, kMlpH);
    const int B = (int)std::min<long long>(batch, n);
    DevBuf db;
    float *dX = db.get<float>((size_t)n * kMlpIn), *dY = db.get<float>(n);
    int *dperm = db.get<int>(n);
    float *p = db.get<float>(kNParam), *gp = db.get<float>(kNParam), *m1 = db.get<float>(kNParam),
          *m2 = db.get<float>(kNParam);
    float *dmean = db.get<float>(kMlpIn), *drstd = db.get<float>(kMlpIn);
    float *x = db.get<float>((size_t)B * kMlpIn), *yt = db.get<float>(B);
    const int nLoss = (B + 255) / 256;
    float *loss = db.get<float>(nLoss);
    MlpBatch act;
    const bool actOk = mlp_batch_alloc(db, B, act);
    if (!dX || !dY || !dperm || !p || !gp || !m1 || !m2 || !dmean || !drstd || !x || !yt || !loss || !actOk)
        return (int)cudaErrorMemoryAllocation;
    cudaMemcpyAsync(dX, X, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dY, Y, sizeof(float) * n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(p, prm.data(), sizeof(float) * kNParam, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dmean, mean, sizeof(float) * kMlpIn, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(drstd, rstd, sizeof(float) * kMlpIn, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(m1, 0, sizeof(float) * kNParam, s);
    cudaMemsetAsync(m2, 0, sizeof(float) * kNParam, s);
    std::vector<int> perm(n);
    for (long long i = 0; i < n; ++i) perm[i] = (int)i;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const int H = kMlpH;
    long long stepCount = 0;
    std::vector<float> lossHost(nLoss);
    for (int ep = 0; ep < epochs; ++ep) {
        for (long long i = n - 1; i > 0; --i) std::swap(perm[i], perm[splitmix(rs) % (uint64_t)(i + 1)]);
        cudaMemcpyAsync(dperm, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(loss, 0, sizeof(float) * nLoss, s);
        for (long long off = 0; off + B <= n; off += B) {
            mlp_gather_kernel<<<(B + 255) / 256, 256, 0, s>>>(B, dperm, (int)off, dX, dY, x, yt, dmean, drstd,
                                                              1.0f / tscale);
            mlp_forward_backward(p, gp, x, yt, B, act, loss, s);
            ++stepCount;
            const float c1 = 1.0f - std::pow(b1, (float)stepCount), c2 = 1.0f - std::pow(b2, (float)stepCount);
            mlp_adam_kernel<<<(kNParam + 255) / 256, 256, 0, s>>>(kNParam, p, gp, m1, m2, lr, b1, b2, eps, c1, c2);
        }
        cudaMemcpyAsync(lossHost.data(), loss, sizeof(float) * nLoss, cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        double lh = 0.0;
        for (int i = 0; i < nLoss; ++i) lh += lossHost[i];
        lastLoss = lh / (double)((n / B) * B);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    cudaMemcpyAsync(prm.data(), p, sizeof(float) * kNParam, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return (int)cudaGetLastError();
    std::memcpy(wts.w1, &prm[kOffW1], sizeof(float) * kNW1);
    std::memcpy(wts.b1, &prm[kOffB1], sizeof(float) * H);
    std::memcpy(wts.w2, &prm[kOffW2], sizeof(float) * kNW2);
    std::memcpy(wts.b2, &prm[kOffB2], sizeof(float) * H);
    std::memcpy(wts.w3, &prm[kOffW3], sizeof(float) * kNW3);
    std::memcpy(wts.b3, &prm[kOffB3], sizeof(float) * H);
    std::memcpy(wts.w4, &prm[kOffW4], sizeof(float) * H);
    wts.b4 = prm[kOffB4];
    return 0;
}

// Mean squared error of one batch and its gradient with respect to the flat
// parameter vector, by the training kernels above (x: standardised inputs,
// y: scaled targets).  0 on success, else a CUDA error.
int mlp_loss_grad(const float *params, const float *x, const float *y, int B, float *grad, double &lossOut,
                  cudaStream_t s)
{
    if (B < 1) return -1;
    DevBuf db;
    const int nLoss = (B + 255) / 256;
    float *p = db.get<float>(kNParam), *gp = db.get<float>(kNParam), *dx = db.get<float>((size_t)B * kMlpIn),
          *dy = db.get<float>(B), *loss = db.get<float>(nLoss);
    MlpBatch act;
    if (!mlp_batch_alloc(db, B, act) || !p || !gp || !dx || !dy || !loss) return (int)cudaErrorMemoryAllocation;
    cudaMemcpyAsync(p, params, sizeof(float) * kNParam, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dx, x, sizeof(float) * B * kMlpIn, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dy, y, sizeof(float) * B, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(loss, 0, sizeof(float) * nLoss, s);
    mlp_forward_backward(p, gp, dx, dy, B, act, loss, s);
    std::vector<float> lh(nLoss);
    cudaMemcpyAsync(grad, gp, sizeof(float) * kNParam, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(lh.data(), loss, sizeof(float) * nLoss, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return (int)cudaGetLastError();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    double acc = 0.0;
    for (int i = 0; i < nLoss; ++i) acc += lh[i];
    lossOut = acc / B;
    return 0;
}

int mlp_param_count() { return kNParam; }

// Byte offset of element (n, k) of a K-major core-matrix tile with `kchunks`
// 8-element K chunks.
static size_t core_offset(int n, int k, int kchunks)
{
    return (size_t)(n >> 3) * (kchunks * 128) + (size_t)(k >> 3) * 128 + (size_t)(n & 7) * 16 + (size_t)(k & 7) * 2;
}

// FP16 weights in the MMA layout (w1: 64 x 16 with K 6..15 zero; w2, w3: 64 x 64).
void mlp_pack(const MlpHostWeights &w, std::vector<uint16_t> &w1c, std::vector<uint16_t> &w2c,
              std::vector<uint16_t> &w3c)
{
    auto bf = [](float f) {
        const __half b = __float2half_rn(f);
        uint16_t u;
        std::memcpy(&u, &b, 2);
        return u;
    };
    w1c.assign(kMlpH * kMlpK1, 0);
    w2c.assign(kMlpH * kMlpH, 0);
    w3c.assign(kMlpH * kMlpH, 0);
    for (int n = 0; n < kMlpH; ++n) {
        for (int k = 0; k < kMlpIn; ++k) w1c[core_offset(n, k, kMlpK1 / 8) / 2] = bf(w.w1[n * kMlpIn + k]);
        for (int k = 0; k < kMlpH; ++k) {
            w2c[core_offset(n, k, kMlpH / 8) / 2] = bf(w.w2[n * kMlpH + k]);
            w3c[core_offset(n, k, kMlpH / 8) / 2] = bf(w.w3[n * kMlpH + k]);
        }
    }
}

template void launch_mlp_source<double>(const DevGrid &, const NsConst &, const Work<double> &,
                                        const TurbWork<double> &, const MlpDev &, Reduce *, unsigned long long *, int,
                                        cudaStream_t);
template void launch_mlp_source<float>(const DevGrid &, const NsConst &, const Work<float> &, const TurbWork<float> &,
                                       const MlpDev &, Reduce *, unsigned long long *, int, cudaStream_t);
template void launch_mlp_capture<double>(const DevGrid &, const NsConst &, const Work<double> &,
                                         const TurbWork<double> &, float *, float *, int *, float *, long long,
                                         unsigned long long *, cudaStream_t);
template void launch_mlp_capture<float>(const DevGrid &, const NsConst &, const Work<float> &, const TurbWork<float> &,
                                        float *, float *, int *, float *, long long, unsigned long long *,
                                        cudaStream_t);

}  // namespace phx
