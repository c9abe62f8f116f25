// mlp.cu -- the warm-start network: a small MLP (dims[0] -> ... -> dims[L],
// GELU between layers) trained and evaluated on the GPU by this file's own
// kernels.  New, no reference counterpart.
//
// Every matrix product is one tcgen05 kernel (k_gemm_bf16<BN>):
//     D[M x N] (FP32) = A[M x K] (BF16) * B[N x K]^T (BF16) (+ bias[N])
// with both operands K-major (row-major with K contiguous).  A CTA owns a
// 128-row x BN-column tile (BN = 64, 128 or 256, chosen per product so that
// small products still spread over many SMs).  K streams through a ring of
// GM_STAGES shared-memory stages, 64 elements (one 128-byte row) at a time:
// one thread issues two tiled tensor copies per stage (A's 128 x 64 box and
// B's BN x 64 box, 128-byte swizzle, rows past M / N and columns past K read
// as zero), waits for the stage, issues four tcgen05.mma (kind::f16, BF16 in,
// FP32 accumulator in TMEM) and commits them to the stage's "empty" barrier;
// the stage is refilled as soon as the products that read it have finished,
// so the copies of the next stages overlap the tensor-core work.  The four
// warps then read the accumulator back with tcgen05.ld (warp w owns TMEM
// lanes 32w..32w+31) and store D.
//
// Training keeps FP32 master weights and BF16 copies in both layouts
// (W [N x Kp] for the forward product, W^T [Kp x N] for the input gradient),
// and writes activations and output gradients in both layouts too, so every
// product -- forward, input gradient, weight gradient -- is the same K-major
// kernel.  The optimiser is AdamW.  Reductions (bias gradients, the loss) are
// fixed-order, so a training run is deterministic.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <vector>

#include "force_pipe.cuh"

namespace tlfea {

constexpr int MLP_TM = 128;    // rows per CTA (the MMA's M)
constexpr int GM_BK = 64;      // K elements per stage: one 128-byte swizzle row
constexpr int GM_STAGES = 4;   // shared-memory ring depth
constexpr int GM_GROUP = 16;   // row tiles per group of the tile order

template <int BN>
struct GemmGeom {
    static constexpr uint32_t A_BYTES = MLP_TM * GM_BK * 2;
    static constexpr uint32_t B_BYTES = BN * GM_BK * 2;
    static constexpr uint32_t STAGE = A_BYTES + B_BYTES;  // a multiple of 1024 (swizzle atoms stay aligned)
    static constexpr size_t SMEM = 1024 + (size_t)GM_STAGES * STAGE;  // + slack to align the ring to 1024 B
};

struct GemmArgs {
    int M, N, K;
    const __nv_bfloat16* A;
    int lda;
    const __nv_bfloat16* B;
    int ldb;
    const float* bias;
    float* D;
    int ldd;
    int* err;
};

// Shared-memory matrix descriptor of a K-major operand in the 128-byte swizzle
// layout that the tensor copies write: rows of 128 bytes, 8-row groups 1024
// bytes apart (stride byte offset), descriptor version 1, swizzle mode 2
// (128 bytes).  The leading byte offset is unused for this layout.  A K step
// of 16 elements inside the 128-byte row advances the start address by 32 B.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Tiled 2-D tensor copy global -> shared (box given by the tensor map), completion
// counted on `bar`; x is the K coordinate (a multiple of 64 here, so 128-byte aligned).
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

template <int BN>
__global__ void __launch_bounds__(128) k_gemm_bf16(const __grid_constant__ CUtensorMap ta,
                                                   const __grid_constant__ CUtensorMap tb, GemmArgs g) {
    using G = GemmGeom<BN>;
    extern __shared__ unsigned char gemm_smem[];
    __shared__ __align__(8) unsigned long long bars[2 * GM_STAGES + 1];  // full[S], empty[S], done
    __shared__ uint32_t tmem_sh;
    __shared__ int ok_sh;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    // grouped tile order: consecutive CTAs walk GM_GROUP row tiles down one
    // column tile before moving right, so the CTAs resident at one time share a
    // few A row panels and B column panels in L2
    const int mtiles = (g.M + MLP_TM - 1) / MLP_TM, ntiles = (g.N + BN - 1) / BN;
    const int per_group = GM_GROUP * ntiles, grp = blockIdx.x / per_group;
    const int first_m = grp * GM_GROUP, gm = min(mtiles - first_m, GM_GROUP);
    const int in_grp = blockIdx.x - grp * per_group;
    const int m0 = (first_m + in_grp % gm) * MLP_TM, n0 = (in_grp / gm) * BN;
    const int nk = (g.K + GM_BK - 1) / GM_BK;
    const uint32_t ring = (smem_u32(gemm_smem) + 1023u) & ~1023u;
    const uint32_t bar0 = smem_u32(bars), done = bar0 + 16 * GM_STAGES;
    auto full = [&](int s) { return bar0 + 8 * s; };
    auto empty = [&](int s) { return bar0 + 8 * (GM_STAGES + s); };
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                     "n"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) {
        for (int i = 0; i < 2 * GM_STAGES + 1; ++i) mbar_init(bar0 + 8 * i, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_sh;
    if (warp == 0) {
        if (lane == 0) {
            // one thread: copies into the ring and tensor-core issue
            constexpr uint32_t idesc = umma_idesc_bf16(MLP_TM, BN);
            bool ok = true;
            int loaded = 0, landed = 0;
            auto load = [&](int k) {
                const int s = k % GM_STAGES;
                const uint32_t a = ring + s * G::STAGE;
                mbar_expect_tx(full(s), G::STAGE);
                tma_load_2d(a, &ta, k * GM_BK, m0, full(s));
                tma_load_2d(a + G::A_BYTES, &tb, k * GM_BK, n0, full(s));
            };
            for (; loaded < nk && loaded < GM_STAGES; ++loaded) load(loaded);
            for (int k = 0; k < nk; ++k) {
                const int s = k % GM_STAGES;
                if (!mbar_wait(full(s), (k / GM_STAGES) & 1)) {
                    ok = false;
                    break;
                }
                landed = k + 1;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a = ring + s * G::STAGE, b = a + G::A_BYTES;
#pragma unroll
                for (int kk = 0; kk < GM_BK / 16; ++kk) {
                    const uint64_t ad = umma_desc_sw128(a + 32 * kk), bd = umma_desc_sw128(b + 32 * kk);
                    const uint32_t acc = (k > 0 || kk > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                        "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                        : "memory");
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 empty(s))
                             : "memory");
                // refill the stage that the previous chunk's products read (they have
                // had this chunk's issue time to finish; the tensor pipe keeps a queue)
                if (k >= 1 && loaded < nk) {
                    const int sp = (k - 1) % GM_STAGES;
                    if (!mbar_wait(empty(sp), ((k - 1) / GM_STAGES) & 1)) {
                        ok = false;
                        break;
                    }
                    load(loaded++);
                }
            }
            // arrives once every product issued above has completed
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(done)
                         : "memory");
            if (!ok) {
                atomicExch(g.err, 5);
                // copies still in flight land before the CTA's shared memory is released
                for (int k = landed; k < loaded; ++k) mbar_wait(full(k % GM_STAGES), (k / GM_STAGES) & 1);
            }
            ok_sh = ok ? 1 : 0;
        }
        __syncwarp();
    }
    const bool got = mbar_wait(done, 0);
    const bool ok = __syncthreads_and(got) && ok_sh;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
        const int row = m0 + warp * 32 + lane;
        const int ncols = min(BN, g.N - n0);
        for (int c0 = 0; c0 < ncols; c0 += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(taddr)
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < g.M) {
                float* d = g.D + (size_t)row * g.ldd + n0 + c0;
                const float* bias = g.bias ? g.bias + n0 + c0 : nullptr;
                const int nc = min(16, ncols - c0);  // N is a multiple of 16, so nc is 16
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (i < nc) d[i] = __uint_as_float(v[i]) + (bias ? bias[i] : 0.f);
            }
        }
    } else if (t == 0) {
        atomicExch(g.err, 5);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(BN) : "memory");
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

// Tensor map of a row-major BF16 operand [rows x k] with leading dimension ld
// (elements): boxes of box_rows x 64, 128-byte swizzle, out-of-range elements
// read as zero.
static int operand_map(CUtensorMap* map, const __nv_bfloat16* base, int rows, int k, int ld, int box_rows) {
    auto enc = tensor_map_encoder();
    if (!enc) {
        set_error("mlp gemm: cuTensorMapEncodeTiled is not available from the driver");
        return TLFEA_CUDA_ERROR;
    }
    const cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)GM_BK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(base), dims, strides,
                           box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("mlp gemm: tensor map encoding failed");
        return TLFEA_INVALID_ARG;
    }
    return TLFEA_OK;
}

// Column-tile width: the widest of 256 / 128 / 64 whose grid still covers the SMs
// (or 64 when even that does not).
static int gemm_tile_n(int M, int N, int sms) {
    const int mt = (M + MLP_TM - 1) / MLP_TM;
    for (int bn : {256, 128})
        if ((long long)mt * ((N + bn - 1) / bn) >= sms) return bn;
    return 64;
}

template <int BN>
static int gemm_launch_bn(const GemmArgs& g, const CUtensorMap& ta, const CUtensorMap& tb, cudaStream_t st) {
    // the shared-memory limit is a per-device attribute of the function: set it once per device
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    TLFEA_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured.load() & bit)) {
        TLFEA_CUDA(cudaFuncSetAttribute(k_gemm_bf16<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)GemmGeom<BN>::SMEM));
        configured.fetch_or(bit);
    }
    const unsigned tiles = (unsigned)(((g.M + MLP_TM - 1) / MLP_TM) * ((g.N + BN - 1) / BN));
    k_gemm_bf16<BN><<<tiles, 128, GemmGeom<BN>::SMEM, st>>>(ta, tb, g);
    TLFEA_CHECK_LAUNCH();
    return TLFEA_OK;
}

static int gemm_launch(const GemmArgs& g, cudaStream_t st) {
    if (g.M <= 0 || g.N <= 0 || g.K <= 0 || g.N % 16 || g.K % 16 || g.lda % 8 || g.ldb % 8 || g.lda < g.K ||
        g.ldb < g.K || (reinterpret_cast<uintptr_t>(g.A) & 15) || (reinterpret_cast<uintptr_t>(g.B) & 15)) {
        set_error("mlp gemm: need N, K multiples of 16, leading dimensions >= K and multiples of 8, 16-byte "
                  "aligned operands");
        return TLFEA_INVALID_ARG;
    }
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    const int bn = gemm_tile_n(g.M, g.N, sms);
    CUtensorMap ta, tb;
    int s = operand_map(&ta, g.A, g.M, g.K, g.lda, MLP_TM);
    if (!s) s = operand_map(&tb, g.B, g.N, g.K, g.ldb, bn);
    if (s) return s;
    if (bn == 256) return gemm_launch_bn<256>(g, ta, tb, st);
    if (bn == 128) return gemm_launch_bn<128>(g, ta, tb, st);
    return gemm_launch_bn<64>(g, ta, tb, st);
}

// ------------------------------------------------------------- elementwise

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float x) {
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// Input rows (FP32, din wide) -> BF16 [B x Kp] (zero padded) and its transpose [Kp x ldT].
__global__ void k_mlp_input(int B, int din, int Kp, const float* __restrict__ X, __nv_bfloat16* H,
                            __nv_bfloat16* HT, int ldT) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * Kp) return;
    const int b = i / Kp, k = i - b * Kp;
    const __nv_bfloat16 v = __float2bfloat16_rn(k < din ? X[(size_t)b * din + k] : 0.f);
    H[i] = v;
    HT[(size_t)k * ldT + b] = v;
}

// H = GELU(Z) as BF16 in both layouts.
__global__ void k_mlp_act(int B, int N, const float* __restrict__ Z, __nv_bfloat16* H, __nv_bfloat16* HT, int ldT) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * N) return;
    const int b = i / N, n = i - b * N;
    const __nv_bfloat16 v = __float2bfloat16_rn(gelu(Z[i]));
    H[i] = v;
    if (HT) HT[(size_t)n * ldT + b] = v;
}

// Mean squared error over B x N: dY = 2 (Y - T) / (B N) in FP32 and BF16 (both
// layouts); per-block partial losses.
__global__ void k_mlp_loss(int B, int N, const float* __restrict__ Y, const float* __restrict__ T, float* dZ,
                           __nv_bfloat16* dZ16, __nv_bfloat16* dZt16, int ldT, float* part) {
    __shared__ float red[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (i < B * N) {
        const int b = i / N, n = i - b * N;
        const float e = Y[i] - T[i];
        const float scale = 1.0f / ((float)B * (float)N);
        l = e * e * scale;
        const float d = 2.0f * e * scale;
        dZ[i] = d;
        const __nv_bfloat16 h = __float2bfloat16_rn(d);
        dZ16[i] = h;
        dZt16[(size_t)n * ldT + b] = h;
    }
    const float s = block_sum(l, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_mlp_sum(int n, const float* __restrict__ part, float* out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        float s = 0.f;
        for (int i = 0; i < n; ++i) s += part[i];
        *out = s;
    }
}

// dZ = dH * GELU'(Z): FP32, and BF16 in both layouts.
__global__ void k_mlp_gelu_back(int B, int N, const float* __restrict__ dH, int ldh, const float* __restrict__ Z,
                                float* dZ, __nv_bfloat16* dZ16, __nv_bfloat16* dZt16, int ldT) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * N) return;
    const int b = i / N, n = i - b * N;
    const float d = dH[(size_t)b * ldh + n] * gelu_grad(Z[i]);
    dZ[i] = d;
    const __nv_bfloat16 h = __float2bfloat16_rn(d);
    dZ16[i] = h;
    dZt16[(size_t)n * ldT + b] = h;
}

// Bias gradient: column sums over the batch, fixed order.
__global__ void k_mlp_colsum(int B, int N, const float* __restrict__ dZ, float* gb) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int b = 0; b < B; ++b) s += dZ[(size_t)b * N + n];
    gb[n] = s;
}

// AdamW on an [N x Kreal] weight (stored with Kp columns) or a bias (Kp = 0),
// bias-corrected moments; refreshes the BF16 copies W [N x Kp] and W^T [Kp x N].
__global__ void k_mlp_adamw(int N, int Kreal, int Kp, float* W, const float* __restrict__ G, int ldg, float* m,
                            float* v, __nv_bfloat16* W16, __nv_bfloat16* Wt16, float lr, float b1, float b2, float eps,
                            float wd, float c1, float c2) {
    const int cols = Kp > 0 ? Kp : 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * cols) return;
    const int n = i / cols, k = i - n * cols;
    if (Kp > 0 && k >= Kreal) return;  // padding stays zero
    const float g = G[(size_t)n * ldg + k];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    float w = W[i];
    w -= lr * (wd * w + (mi / c1) / (sqrtf(vi / c2) + eps));
    W[i] = w;
    if (W16) {
        const __nv_bfloat16 h = __float2bfloat16_rn(w);
        W16[i] = h;
        Wt16[(size_t)k * N + n] = h;
    }
}

__global__ void k_mlp_to_bf16(int N, int Kp, const float* __restrict__ W, __nv_bfloat16* W16, __nv_bfloat16* Wt16) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * Kp) return;
    const int n = i / Kp, k = i - n * Kp;
    const __nv_bfloat16 h = __float2bfloat16_rn(W[i]);
    W16[i] = h;
    Wt16[(size_t)k * N + n] = h;
}

}  // namespace tlfea

using namespace tlfea;

struct tlfea_mlp_s {
    int L = 0;
    std::vector<int> dims, Kp, Np;  // Kp: padded input width, Np: output rows padded to 128
    int Bmax = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    int* err = nullptr;
    std::vector<float*> W, b, mW, vW, mb, vb, gW, gb, Z;
    std::vector<__nv_bfloat16*> W16, Wt16, H, HT;  // H[l], HT[l]: input of layer l
    float *dZ = nullptr, *dH = nullptr, *part = nullptr, *loss = nullptr, *xin = nullptr, *tin = nullptr;
    __nv_bfloat16 *dZ16 = nullptr, *dZt16 = nullptr;
    int maxN = 0, maxK = 0, maxNp = 0;
    long long step = 0;
    bool grads_valid = false;
};

namespace {

int mlp_check_err(tlfea_mlp_s* m) {
    int e = 0;
    TLFEA_CUDA(cudaMemcpyAsync(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    TLFEA_CUDA(cudaStreamSynchronize(m->stream));
    if (e) {
        cudaMemsetAsync(m->err, 0, sizeof(int), m->stream);
        set_error("mlp: a tensor-core product did not complete (bounded wait ran out)");
        return TLFEA_CUDA_ERROR;
    }
    return TLFEA_OK;
}

inline unsigned grid1(long long n, int bs = 256) { return (unsigned)((n + bs - 1) / bs); }

int mlp_forward(tlfea_mlp_s* m, const float* X, int B, bool keep_transposes) {
    cudaStream_t st = m->stream;
    k_mlp_input<<<grid1((long long)B * m->Kp[0]), 256, 0, st>>>(B, m->dims[0], m->Kp[0], X, m->H[0], m->HT[0], m->Bmax);
    TLFEA_CHECK_LAUNCH();
    for (int l = 0; l < m->L; ++l) {
        GemmArgs g{B, m->dims[l + 1], m->Kp[l], m->H[l], m->Kp[l], m->W16[l], m->Kp[l], m->b[l], m->Z[l],
                   m->dims[l + 1], m->err};
        int s = gemm_launch(g, st);
        if (s) return s;
        if (l + 1 < m->L) {
            const int N = m->dims[l + 1];
            k_mlp_act<<<grid1((long long)B * N), 256, 0, st>>>(B, N, m->Z[l], m->H[l + 1],
                                                               keep_transposes ? m->HT[l + 1] : nullptr, m->Bmax);
            TLFEA_CHECK_LAUNCH();
        }
    }
    return TLFEA_OK;
}

int mlp_backward(tlfea_mlp_s* m, const float* T, int B) {
    cudaStream_t st = m->stream;
    const int L = m->L;
    const int Nout = m->dims[L];
    const unsigned nb = grid1((long long)B * Nout);
    k_mlp_loss<<<nb, 256, 0, st>>>(B, Nout, m->Z[L - 1], T, m->dZ, m->dZ16, m->dZt16, m->Bmax, m->part);
    TLFEA_CHECK_LAUNCH();
    k_mlp_sum<<<1, 32, 0, st>>>((int)nb, m->part, m->loss);
    TLFEA_CHECK_LAUNCH();
    for (int l = L - 1; l >= 0; --l) {
        const int N = m->dims[l + 1];
        // weight gradient: gW[Np x Kp] = dZ^T (rows padded with zeros) x H
        GemmArgs gw{m->Np[l], m->Kp[l], B, m->dZt16, m->Bmax, m->HT[l], m->Bmax, nullptr, m->gW[l], m->Kp[l], m->err};
        int s = gemm_launch(gw, st);
        if (s) return s;
        k_mlp_colsum<<<grid1(N, 128), 128, 0, st>>>(B, N, m->dZ, m->gb[l]);
        TLFEA_CHECK_LAUNCH();
        if (l == 0) break;
        // input gradient: dH[B x Kp] = dZ x W (= dZ x (W^T)^T)
        GemmArgs gx{B, m->Kp[l], N, m->dZ16, N, m->Wt16[l], N, nullptr, m->dH, m->Kp[l], m->err};
        if ((s = gemm_launch(gx, st))) return s;
        const int Nprev = m->dims[l];
        k_mlp_gelu_back<<<grid1((long long)B * Nprev), 256, 0, st>>>(B, Nprev, m->dH, m->Kp[l], m->Z[l - 1], m->dZ,
                                                                     m->dZ16, m->dZt16, m->Bmax);
        TLFEA_CHECK_LAUNCH();
    }
    return TLFEA_OK;
}

int mlp_adamw(tlfea_mlp_s* m, float lr, float b1, float b2, float eps, float wd) {
    cudaStream_t st = m->stream;
    m->step += 1;
    const float c1 = 1.0f - powf(b1, (float)m->step), c2 = 1.0f - powf(b2, (float)m->step);
    for (int l = 0; l < m->L; ++l) {
        const int N = m->dims[l + 1], K = m->dims[l], Kp = m->Kp[l];
        k_mlp_adamw<<<grid1((long long)N * Kp), 256, 0, st>>>(N, K, Kp, m->W[l], m->gW[l], Kp, m->mW[l], m->vW[l],
                                                              m->W16[l], m->Wt16[l], lr, b1, b2, eps, wd, c1, c2);
        TLFEA_CHECK_LAUNCH();
        k_mlp_adamw<<<grid1(N), 256, 0, st>>>(N, 1, 0, m->b[l], m->gb[l], 1, m->mb[l], m->vb[l], nullptr, nullptr, lr,
                                              b1, b2, eps, 0.f, c1, c2);
        TLFEA_CHECK_LAUNCH();
    }
    return TLFEA_OK;
}

int mlp_refresh_bf16(tlfea_mlp_s* m) {
    for (int l = 0; l < m->L; ++l) {
        const int N = m->dims[l + 1], Kp = m->Kp[l];
        k_mlp_to_bf16<<<grid1((long long)N * Kp), 256, 0, m->stream>>>(N, Kp, m->W[l], m->W16[l], m->Wt16[l]);
        TLFEA_CHECK_LAUNCH();
    }
    return TLFEA_OK;
}

long long mlp_param_count(const tlfea_mlp_s* m) {
    long long n = 0;
    for (int l = 0; l < m->L; ++l) n += (long long)m->dims[l + 1] * m->dims[l] + m->dims[l + 1];
    return n;
}

}  // namespace

#define CHECK_MLP(m)                  \
    do {                              \
        if (!(m)) {                   \
            set_error("null mlp");    \
            return TLFEA_INVALID_ARG; \
        }                             \
    } while (0)

extern "C" {

int tlfea_mlp_gemm_bf16(int M, int N, int K, const void* d_a, int lda, const void* d_b, int ldb, const float* d_bias,
                        float* d_d, int ldd, void* stream) {
    int* err = nullptr;
    int s = dalloc(&err, 1);
    if (s) return s;
    cudaStream_t st = (cudaStream_t)stream;
    TLFEA_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    GemmArgs g{M, N, K, (const __nv_bfloat16*)d_a, lda, (const __nv_bfloat16*)d_b, ldb, d_bias, d_d, ldd, err};
    s = gemm_launch(g, st);
    int e = 0;
    if (!s && cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
        cudaStreamSynchronize(st) == cudaSuccess && e) {
        set_error("mlp gemm: bounded wait ran out");
        s = TLFEA_CUDA_ERROR;
    }
    cudaStreamSynchronize(st);
    dfree(err);
    return s;
}

int tlfea_mlp_gemm_bf16_async(int M, int N, int K, const void* d_a, int lda, const void* d_b, int ldb,
                              const float* d_bias, float* d_d, int ldd, int* d_err, void* stream) {
    if (!d_err || !d_d) {
        set_error("mlp gemm: null output or error flag");
        return TLFEA_INVALID_ARG;
    }
    GemmArgs g{M, N, K, (const __nv_bfloat16*)d_a, lda, (const __nv_bfloat16*)d_b, ldb, d_bias, d_d, ldd, d_err};
    return gemm_launch(g, (cudaStream_t)stream);
}

int tlfea_mlp_create(int n_layers, const int* dims, int max_batch, unsigned long long seed, tlfea_mlp* out) {
    if (!out || !dims || n_layers < 1 || max_batch <= 0 || max_batch % 128) {
        set_error("mlp_create: need >= 1 layer and max_batch a positive multiple of 128");
        return TLFEA_INVALID_ARG;
    }
    for (int l = 1; l <= n_layers; ++l)
        if (dims[l] <= 0 || dims[l] % 16 || dims[l] > 4096) {
            set_error("mlp_create: layer widths must be positive multiples of 16 (<= 4096)");
            return TLFEA_INVALID_ARG;
        }
    if (dims[0] <= 0 || dims[0] > 4096) return TLFEA_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_error("no CUDA device");
        return TLFEA_NO_CUDA_DEVICE;
    }
    tlfea_mlp_s* m = new tlfea_mlp_s();
    cudaGetDevice(&m->device);
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete m;
        set_error("cudaStreamCreate failed");
        return TLFEA_CUDA_ERROR;
    }
    m->L = n_layers;
    m->dims.assign(dims, dims + n_layers + 1);
    m->Bmax = max_batch;
    for (int l = 0; l < n_layers; ++l) {
        m->Kp.push_back((dims[l] + 15) / 16 * 16);
        m->Np.push_back((dims[l + 1] + MLP_TM - 1) / MLP_TM * MLP_TM);
        m->maxN = std::max(m->maxN, dims[l + 1]);
        m->maxK = std::max(m->maxK, m->Kp[l]);
        m->maxNp = std::max(m->maxNp, m->Np[l]);
    }
    const int L = n_layers, B = max_batch;
    m->W.assign(L, nullptr); m->b.assign(L, nullptr); m->mW.assign(L, nullptr); m->vW.assign(L, nullptr);
    m->mb.assign(L, nullptr); m->vb.assign(L, nullptr); m->gW.assign(L, nullptr); m->gb.assign(L, nullptr);
    m->Z.assign(L, nullptr); m->W16.assign(L, nullptr); m->Wt16.assign(L, nullptr);
    m->H.assign(L, nullptr); m->HT.assign(L, nullptr);
    int s = dalloc(&m->err, 1);
    for (int l = 0; l < L && !s; ++l) {
        const size_t nk = (size_t)dims[l + 1] * m->Kp[l];
        s = dalloc(&m->W[l], nk) | dalloc(&m->mW[l], nk) | dalloc(&m->vW[l], nk) |
            dalloc(&m->gW[l], (size_t)m->Np[l] * m->Kp[l]) | dalloc(&m->b[l], dims[l + 1]) |
            dalloc(&m->mb[l], dims[l + 1]) | dalloc(&m->vb[l], dims[l + 1]) | dalloc(&m->gb[l], dims[l + 1]) |
            dalloc(&m->Z[l], (size_t)B * dims[l + 1]) | dalloc(&m->W16[l], nk) | dalloc(&m->Wt16[l], nk) |
            dalloc(&m->H[l], (size_t)B * m->Kp[l]) | dalloc(&m->HT[l], (size_t)m->Kp[l] * B);
    }
    if (!s)
        s = dalloc(&m->dZ, (size_t)B * m->maxN) | dalloc(&m->dH, (size_t)B * m->maxK) |
            dalloc(&m->dZ16, (size_t)B * m->maxN) | dalloc(&m->dZt16, (size_t)m->maxNp * B) |
            dalloc(&m->part, (size_t)(B * m->maxN + 255) / 256 + 1) | dalloc(&m->loss, 1) |
            dalloc(&m->xin, (size_t)B * dims[0]) | dalloc(&m->tin, (size_t)B * dims[L]);
    if (s) {
        tlfea_mlp_destroy(m);
        return TLFEA_CUDA_ERROR;
    }
    // zero everything the padding relies on (padded weight columns, padded
    // gradient rows), then a seeded uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) init
    cudaStream_t st = m->stream;
    cudaMemsetAsync(m->err, 0, sizeof(int), st);
    cudaMemsetAsync(m->dZt16, 0, (size_t)m->maxNp * B * sizeof(__nv_bfloat16), st);
    for (int l = 0; l < L; ++l) {
        const size_t nk = (size_t)dims[l + 1] * m->Kp[l];
        cudaMemsetAsync(m->mW[l], 0, nk * 4, st);
        cudaMemsetAsync(m->vW[l], 0, nk * 4, st);
        cudaMemsetAsync(m->mb[l], 0, dims[l + 1] * 4, st);
        cudaMemsetAsync(m->vb[l], 0, dims[l + 1] * 4, st);
        cudaMemsetAsync(m->H[l], 0, (size_t)B * m->Kp[l] * 2, st);
        cudaMemsetAsync(m->HT[l], 0, (size_t)m->Kp[l] * B * 2, st);
    }
    std::vector<float> flat((size_t)mlp_param_count(m));
    unsigned long long x = seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    auto next = [&]() {  // splitmix64
        x += 0x9E3779B97F4A7C15ull;
        unsigned long long z = x;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    size_t o = 0;
    for (int l = 0; l < L; ++l) {
        const float bound = 1.0f / std::sqrt((float)dims[l]);
        const size_t cnt = (size_t)dims[l + 1] * dims[l] + dims[l + 1];
        for (size_t i = 0; i < cnt; ++i) flat[o + i] = bound * (2.0f * (float)((next() >> 11) * 0x1.0p-53) - 1.0f);
        o += cnt;
    }
    cudaStreamSynchronize(st);
    s = tlfea_mlp_set_params(m, flat.data(), (long long)flat.size());
    if (s) {
        tlfea_mlp_destroy(m);
        return s;
    }
    *out = m;
    return TLFEA_OK;
}

int tlfea_mlp_destroy(tlfea_mlp m) {
    CHECK_MLP(m);
    TLFEA_CUDA(cudaSetDevice(m->device));
    if (m->stream) cudaStreamSynchronize(m->stream);
    for (auto* v : {&m->W, &m->b, &m->mW, &m->vW, &m->mb, &m->vb, &m->gW, &m->gb, &m->Z})
        for (auto& p : *v) dfree(p);
    for (auto* v : {&m->W16, &m->Wt16, &m->H, &m->HT})
        for (auto& p : *v) dfree(p);
    dfree(m->dZ); dfree(m->dH); dfree(m->part); dfree(m->loss); dfree(m->xin); dfree(m->tin);
    dfree(m->dZ16); dfree(m->dZt16); dfree(m->err);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return TLFEA_OK;
}

int tlfea_mlp_get_stream(tlfea_mlp m, void** stream) {
    CHECK_MLP(m);
    if (!stream) return TLFEA_INVALID_ARG;
    *stream = (void*)m->stream;
    return TLFEA_OK;
}

int tlfea_mlp_param_count(tlfea_mlp m, long long* n) {
    CHECK_MLP(m);
    if (!n) return TLFEA_INVALID_ARG;
    *n = mlp_param_count(m);
    return TLFEA_OK;
}

// Flat FP32 parameters: per layer W [dims[l+1] x dims[l]] row-major, then b.
int tlfea_mlp_set_params(tlfea_mlp m, const float* p, long long n) {
    CHECK_MLP(m);
    if (!p || n != mlp_param_count(m)) {
        set_error("mlp_set_params: size mismatch");
        return TLFEA_SIZE_MISMATCH;
    }
    size_t o = 0;
    for (int l = 0; l < m->L; ++l) {
        const int N = m->dims[l + 1], K = m->dims[l], Kp = m->Kp[l];
        std::vector<float> w((size_t)N * Kp, 0.f);
        for (int r = 0; r < N; ++r)
            for (int k = 0; k < K; ++k) w[(size_t)r * Kp + k] = p[o + (size_t)r * K + k];
        o += (size_t)N * K;
        TLFEA_CUDA(cudaMemcpyAsync(m->W[l], w.data(), w.size() * 4, cudaMemcpyHostToDevice, m->stream));
        TLFEA_CUDA(cudaMemcpyAsync(m->b[l], p + o, (size_t)N * 4, cudaMemcpyHostToDevice, m->stream));
        o += N;
        TLFEA_CUDA(cudaStreamSynchronize(m->stream));
    }
    const int s = mlp_refresh_bf16(m);
    if (s) return s;
    TLFEA_CUDA(cudaStreamSynchronize(m->stream));
    return TLFEA_OK;
}

int tlfea_mlp_get_params(tlfea_mlp m, float* p, long long n) {
    CHECK_MLP(m);
    if (!p || n != mlp_param_count(m)) {
        set_error("mlp_get_params: size mismatch");
        return TLFEA_SIZE_MISMATCH;
    }
    size_t o = 0;
    for (int l = 0; l < m->L; ++l) {
        const int N = m->dims[l + 1], K = m->dims[l], Kp = m->Kp[l];
        std::vector<float> w((size_t)N * Kp);
        TLFEA_CUDA(cudaMemcpyAsync(w.data(), m->W[l], w.size() * 4, cudaMemcpyDeviceToHost, m->stream));
        TLFEA_CUDA(cudaMemcpyAsync(p + o + (size_t)N * K, m->b[l], (size_t)N * 4, cudaMemcpyDeviceToHost, m->stream));
        TLFEA_CUDA(cudaStreamSynchronize(m->stream));
        for (int r = 0; r < N; ++r)
            for (int k = 0; k < K; ++k) p[o + (size_t)r * K + k] = w[(size_t)r * Kp + k];
        o += (size_t)N * K + N;
    }
    return TLFEA_OK;
}

// Gradients of the last loss_grad call, in the parameter layout.
int tlfea_mlp_get_grads(tlfea_mlp m, float* g, long long n) {
    CHECK_MLP(m);
    if (!g || n != mlp_param_count(m)) {
        set_error("mlp_get_grads: size mismatch");
        return TLFEA_SIZE_MISMATCH;
    }
    if (!m->grads_valid) {
        set_error("mlp_get_grads: no gradients computed yet");
        return TLFEA_NOT_SETUP;
    }
    size_t o = 0;
    for (int l = 0; l < m->L; ++l) {
        const int N = m->dims[l + 1], K = m->dims[l], Kp = m->Kp[l];
        std::vector<float> w((size_t)m->Np[l] * Kp);
        TLFEA_CUDA(cudaMemcpyAsync(w.data(), m->gW[l], w.size() * 4, cudaMemcpyDeviceToHost, m->stream));
        TLFEA_CUDA(cudaMemcpyAsync(g + o + (size_t)N * K, m->gb[l], (size_t)N * 4, cudaMemcpyDeviceToHost, m->stream));
        TLFEA_CUDA(cudaStreamSynchronize(m->stream));
        for (int r = 0; r < N; ++r)
            for (int k = 0; k < K; ++k) g[o + (size_t)r * K + k] = w[(size_t)r * Kp + k];
        o += (size_t)N * K + N;
    }
    return TLFEA_OK;
}

// y[batch x dims[L]] = MLP(x[batch x dims[0]]), device pointers, on the MLP stream.
int tlfea_mlp_forward(tlfea_mlp m, const float* d_x, int batch, float* d_y) {
    CHECK_MLP(m);
    if (!d_x || !d_y || batch <= 0 || batch > m->Bmax) return TLFEA_INVALID_ARG;
    int s = mlp_forward(m, d_x, batch, false);
    if (s) return s;
    const int Nout = m->dims[m->L];
    TLFEA_CUDA(cudaMemcpyAsync(d_y, m->Z[m->L - 1], (size_t)batch * Nout * 4, cudaMemcpyDeviceToDevice, m->stream));
    return mlp_check_err(m);
}

// Forward + backward of the mean squared error against d_t; keeps the
// gradients; *loss (host) = the batch loss.  batch must be a multiple of 16.
int tlfea_mlp_loss_grad(tlfea_mlp m, const float* d_x, const float* d_t, int batch, float* loss) {
    CHECK_MLP(m);
    if (!d_x || !d_t || batch <= 0 || batch > m->Bmax || batch % 16) {
        set_error("mlp_loss_grad: batch must be a positive multiple of 16 up to max_batch");
        return TLFEA_INVALID_ARG;
    }
    int s = mlp_forward(m, d_x, batch, true);
    if (!s) s = mlp_backward(m, d_t, batch);
    if (s) return s;
    if (loss) TLFEA_CUDA(cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->stream));
    s = mlp_check_err(m);
    if (s) return s;
    m->grads_valid = true;
    return TLFEA_OK;
}

int tlfea_mlp_adamw_step(tlfea_mlp m, float lr, float beta1, float beta2, float eps, float weight_decay) {
    CHECK_MLP(m);
    if (!m->grads_valid) {
        set_error("mlp_adamw_step: no gradients computed yet");
        return TLFEA_NOT_SETUP;
    }
    const int s = mlp_adamw(m, lr, beta1, beta2, eps, weight_decay);
    if (s) return s;
    return TLFEA_OK;
}

// One optimisation step on a minibatch: forward, backward, AdamW.  With
// loss == NULL nothing is read back (no host synchronisation).
int tlfea_mlp_train_step(tlfea_mlp m, const float* d_x, const float* d_t, int batch, float lr, float beta1,
                         float beta2, float eps, float weight_decay, float* loss) {
    CHECK_MLP(m);
    if (!d_x || !d_t || batch <= 0 || batch > m->Bmax || batch % 16) {
        set_error("mlp_train_step: batch must be a positive multiple of 16 up to max_batch");
        return TLFEA_INVALID_ARG;
    }
    int s = mlp_forward(m, d_x, batch, true);
    if (!s) s = mlp_backward(m, d_t, batch);
    if (!s) s = mlp_adamw(m, lr, beta1, beta2, eps, weight_decay);
    if (s) return s;
    m->grads_valid = true;
    if (loss) {
        TLFEA_CUDA(cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->stream));
        return mlp_check_err(m);
    }
    return TLFEA_OK;
}

int tlfea_mlp_sync(tlfea_mlp m) {
    CHECK_MLP(m);
    return mlp_check_err(m);
}

}  // extern "C"
