// The split-BF16 position pass for a 128 x 128 detector: the 2-D DFT pair as products with a real 128 x 128 matrix on
// the tensor cores.
//
// Arithmetic (Ptychography.swift:321-350): exit wave X = S * O[patch], F = fft2(X), the Fourier-modulus projection with
// the 1/n of ifft2 folded in, then dpsi = ifft2(F').  The 128-point DFT matrix factors as W = T C with C real:
//
//   C row 0 = 1, row 1 = cos(pi k), rows 2j and 2j + 1 = cos(2 pi j k / 128) and sin(2 pi j k / 128)  (j = 1..63)
//
// and T combining row pairs: for z = C x, (W x)[j] = z[2j] - i z[2j+1] and (W x)[128 - j] = z[2j] + i z[2j+1]
// ((W x)[0] = z[0], (W x)[64] = z[1]); conj(W) swaps the two.  Every transform is therefore the real product D = C B of
// the re and the im plane separately, half the multiply-adds of a complex DFT matrix, and T is applied only where a
// stage's result is needed in the frequency or pixel basis: on a row of D inside one thread, and between the rows of
// TMEM lanes 2j and 2j + 1 (adjacent lanes of a warp) with one shuffle per value.  With D[m][n] = sum_k A[m][k] B[n][k]
// (A = C or C_sigma in tensor memory, B = data in shared memory):
//
//   stage 1  B[n = r][k = c]   = X                       K-major   D[raw c][r]
//   stage 2  B[n = raw c][k = r] = D1                    K-major   D[raw r][raw c]  -> T both ways -> F[kr][kc]
//   stage 3  B[n = pos][k = kr] = F'[kr][sigma(pos)]     MN-major  D[raw r][pos]
//   stage 4  B[n = raw r][k = pos] = D3, A = C_sigma     K-major   D[raw c][raw r]  -> T both ways -> dpsi[r][c]
//
// sigma orders the frequencies kc the way one thread holds them after T (8 consecutive positions per thread and
// row), and C_sigma[m][pos] = C[m][sigma(pos)] contracts over them in that order.  Each real product P Q is
// P_hi Q_hi + P_hi Q_lo + P_lo Q_hi in bf16 with FP32 accumulation in tensor memory: 3 x 8 K-steps = 24 tcgen05.mma
// (M = N = 128, K = 16) per plane and stage.  The two planes run as a pipeline: the re plane's result is read out and
// its next stage issued while the tensor core still works on the im plane.
//
// One persistent CTA of kThreads = 512 threads per SM with 208 KB of shared memory: the four B planes and the next
// position's amplitudes, bulk-copied in behind stages 3 to 2.  Tensor memory: C hi / lo (columns 0-127), C_sigma hi / lo
// (128-255), the re-plane result (256-383), the im-plane result (384-511).  Thread (warp w, lane i) owns TMEM lane
// 32 (w mod 4) + i and the kCols-column group w / 4 of each result (kCols = 32).  The layout constants follow from
// kThreads; 1024 threads (kCols = 16, 64 registers) measured 8.91 against 8.37 ms per pass of 65,536 positions: the
// phases between the products are bound by instruction issue more than by latency, and twice the warps only add barrier
// cost and spills.  Amplitudes are pre-permuted into the order each thread consumes them (a warp reads 512 contiguous
// bytes per load); dpsi is written [position][row][column].  Waits are bounded: a wait that runs out sets *fault and
// the CTA stops after freeing its tensor memory.
#include "engine.h"
#include "umma.cuh"

namespace cubo {

namespace {

using namespace umma;

constexpr int kN = 128;
constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kGroups = kWarps / 4;        // warps per TMEM lane quadrant: column groups of a result
constexpr int kCols = kN / kGroups;        // result columns per thread (32)
constexpr int kSub = kCols / 16;           // sub-blocks of 4 column pairs per parity set (2)
constexpr int kRowsPerWarp = kN / kWarps;  // exit-wave rows per warp (8)
constexpr int kBatch = 2048 / kThreads;    // exit-wave rows whose loads are in flight at once (4)
static_assert(kCols % 16 == 0 && kRowsPerWarp % kBatch == 0, "thread layout");
// Canonical no-swizzle layout of a 128 x 128 bf16 plane with its core matrices (8 rows x 16 bytes) 144 bytes apart
// along K: the 16 bytes of padding put the K chunks of one row in different banks, so 4-byte stores of consecutive K
// by consecutive lanes (the exit wave) and 16-byte stores of consecutive rows (the other stages) are conflict-free.
constexpr uint32_t kLBO = 144, kSBO = 16 * kLBO;
constexpr int kPlaneBytes = 16 * kSBO;          // 36 KB
constexpr uint64_t kWaitLimit = 2000000000ull;  // ns of wall time an mbarrier wait may take before giving up
constexpr uint32_t kCNat = 0, kCSigma = 128, kSlotRe = 256, kSlotIm = 384;  // tensor-memory columns
constexpr int kReHi = 0, kImHi = 2;             // B planes: re hi, re lo, im hi, im lo
constexpr uint32_t kIdescK = idesc_bf16(128, 128, false, false), kIdescMN = idesc_bf16(128, 128, false, true);

__device__ __forceinline__ uint32_t kmajor_offset(int row, int k) {
    return (row >> 3) * kSBO + (k >> 3) * kLBO + (row & 7) * 16 + (k & 7) * 2;
}
__device__ __forceinline__ uint32_t mnmajor_offset(int k, int col) {
    return (col >> 3) * kSBO + (k >> 3) * kLBO + (k & 7) * 16 + (col & 7) * 2;
}

__device__ __forceinline__ int wrap_once(int v, int size) { return v < 0 ? v + size : (v >= size ? v - size : v); }

// Packed FP32x2 arithmetic (sm_100 mul / fma / sub .f32x2): one instruction for two values, each rounded as the scalar
// operation rounds it.
__device__ __forceinline__ float2 pmul(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

// The frequency paired with j by T: 128 - j, and 64 for j = 0.
__host__ __device__ __forceinline__ int mirror(int j) { return j == 0 ? 64 : kN - j; }

// Writes 8 consecutive K (or MN) values of one row, split into bf16 hi and lo, into planes hi_plane and hi_plane + 1.
__device__ __forceinline__ void store_split8(uint8_t *planes, int hi_plane, uint32_t off, const float (&v)[8]) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; i++) split_bf16x2(v[2 * i], v[2 * i + 1], h[i], l[i]);
    *reinterpret_cast<uint4 *>(planes + hi_plane * kPlaneBytes + off) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4 *>(planes + (hi_plane + 1) * kPlaneBytes + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

// The 24 MMAs of one plane: D (columns d_col) = A (hi at a_col, lo at a_col + 64) * B (planes at b_hi, b_hi + one plane).
__device__ __forceinline__ void issue_plane(uint32_t tmem, uint32_t a_col, uint32_t d_col, uint32_t b_hi, uint32_t idesc) {
#pragma unroll
    for (int s = 0; s < kN / 16; s++) {
        const uint64_t dh = smem_desc(b_hi + s * 2 * kLBO, kLBO, kSBO);
        const uint64_t dl = smem_desc(b_hi + kPlaneBytes + s * 2 * kLBO, kLBO, kSBO);
        mma_ts(tmem + d_col, tmem + a_col + s * 8, dh, idesc, s > 0 ? 1u : 0u);
        mma_ts(tmem + d_col, tmem + a_col + s * 8, dl, idesc, 1u);
        mma_ts(tmem + d_col, tmem + a_col + 64 + s * 8, dh, idesc, 1u);
    }
}

// Lane `row`'s kCols columns of one result (from taddr) -> kCols consecutive K of row `row` of a K-major B plane pair.
__device__ __forceinline__ void readout_kmajor(uint32_t taddr, uint8_t *planes, int hi_plane, int row, int k0) {
    float a[kCols];
#pragma unroll
    for (int c = 0; c < kCols / 16; c++) tmem_ld16(taddr + 16 * c, *reinterpret_cast<float(*)[16]>(a + 16 * c));
    tmem_wait_ld();
#pragma unroll
    for (int c = 0; c < kCols / 8; c++) {
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) v[i] = a[8 * c + i];
        store_split8(planes, hi_plane, kmajor_offset(row, k0 + 8 * c), v);
    }
}

// T on the columns of one lane: raw pairs (zc, zs) = columns (2J, 2J+1) -> the values at J (y0) and mirror(J) (y1).
// Forward: y0 = zc - i zs, y1 = zc + i zs; inverse the other way round; J = 0 passes (z0, z1) through.
template <bool kInverse>
__device__ __forceinline__ void combine(float zr, float zi, float sr, float si, bool passthrough, float &y0r, float &y0i,
                                        float &y1r, float &y1i) {
    if (passthrough) {
        y0r = zr; y0i = zi; y1r = sr; y1i = si;
    } else if (!kInverse) {
        y0r = zr + si; y0i = zi - sr; y1r = zr - si; y1i = zi + sr;
    } else {
        y0r = zr - si; y0i = zi + sr; y1r = zr + si; y1i = zi - sr;
    }
}

// The column index J of a thread's value i (0..3) of sub-block u: its column group g and parity h (= L & 1) own the
// raw result columns kCols g .. kCols g + kCols - 1, i.e. the column pairs (2J, 2J + 1) of J = (kCols / 2) g + 0 ..
// kCols / 2 - 1, of which it keeps, after the exchange with lane L ^ 1, the half of parity h.
__host__ __device__ __forceinline__ int column_of(int g, int h, int u, int i) {
    return (kCols / 2) * g + (kCols / 4) * h + 4 * u + i;
}

// One thread's 16 values of a combined stage result for sub-block u: T on the columns (in the thread), then the
// exchange with lane L ^ 1, then T on the row pair (2j, 2j + 1).  out[side][4 s + i] is the value at row
// (side ? mirror(j) : j) and column (s ? mirror(J) : J), J = column_of(g, h, u, i), h = L & 1.
template <bool kInverse>
__device__ __forceinline__ void combined_block(uint32_t lane_addr, int g, int u, int j, int h, float (&out_re)[2][8],
                                               float (&out_im)[2][8]) {
    float r0[8], r1[8], i0[8], i1[8];  // raw columns of parity sets 0 and 1: kCols g + (kCols / 2) h' + 8 u .. + 8
    tmem_ld8(lane_addr + kSlotRe + kCols * g + 8 * u, r0);
    tmem_ld8(lane_addr + kSlotRe + kCols * g + kCols / 2 + 8 * u, r1);
    tmem_ld8(lane_addr + kSlotIm + kCols * g + 8 * u, i0);
    tmem_ld8(lane_addr + kSlotIm + kCols * g + kCols / 2 + 8 * u, i1);
    tmem_wait_ld();
    // T on the columns for both parity sets: ya / yb [s][i] (complex as re, im)
    float ar[2][4], ai[2][4], br[2][4], bi[2][4];
    const bool first = g == 0 && u == 0;  // J = 0 sits at i = 0 of parity set 0
#pragma unroll
    for (int i = 0; i < 4; i++) {
        combine<kInverse>(r0[2 * i], i0[2 * i], r0[2 * i + 1], i0[2 * i + 1], first && i == 0, ar[0][i], ai[0][i],
                          ar[1][i], ai[1][i]);
        combine<kInverse>(r1[2 * i], i1[2 * i], r1[2 * i + 1], i1[2 * i + 1], false, br[0][i], bi[0][i], br[1][i],
                          bi[1][i]);
    }
    // keep the own parity set, send the other: afterwards `mine` is lane L's row and `theirs` lane L ^ 1's, both for
    // the columns of set h
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float mr = h ? br[s][i] : ar[s][i], mi = h ? bi[s][i] : ai[s][i];
            const float sr = h ? ar[s][i] : br[s][i], si = h ? ai[s][i] : bi[s][i];
            const float tr = __shfl_xor_sync(0xffffffffu, sr, 1), ti = __shfl_xor_sync(0xffffffffu, si, 1);
            // a = row 2j, b = row 2j + 1
            const float a_r = h ? tr : mr, a_i = h ? ti : mi, b_r = h ? mr : tr, b_i = h ? mi : ti;
            float y0r, y0i, y1r, y1i;
            combine<kInverse>(a_r, a_i, b_r, b_i, j == 0, y0r, y0i, y1r, y1i);
            out_re[0][4 * s + i] = y0r; out_im[0][4 * s + i] = y0i;
            out_re[1][4 * s + i] = y1r; out_im[1][4 * s + i] = y1i;
        }
}

__global__ void __launch_bounds__(kThreads, 1) bf16_position_kernel(Bf16Args a) {
    extern __shared__ __align__(1024) uint8_t planes[];  // 4 x 36 KB: the B operand, then 64 KB of amplitudes
    __shared__ uint64_t mbar[2];                         // completion of the re / im plane's MMAs
    __shared__ uint64_t amp_bar;                         // arrival of the next position's amplitudes
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int q = warp & 3, g = warp >> 2;
    const int L = 32 * q + lane;      // this thread's TMEM lane
    const int j = L >> 1, h = L & 1;  // its row pair and parity
    if (warp == 0) {
        tmem_alloc(&tmem_base, 512);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        mbar_init(&amp_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_base;
    const uint32_t lane_addr = tmem_addr(tmem, 32 * q, 0);
    const uint32_t smem = smem_u32(planes);
    float4 *amp_smem = reinterpret_cast<float4 *>(planes + 4 * kPlaneBytes);
    const int last = a.first + a.count;
    bool amp_pending = a.first + (int)blockIdx.x < last;  // a bulk copy of amplitudes is in flight
    if (tid == 0 && amp_pending)
        bulk_load(amp_smem, a.amplitudes + (size_t)(a.first + blockIdx.x) * (kN * kN), kN * kN * 4, &amp_bar);
    uint32_t amp_phase = 0;
    // C hi, C lo, C_sigma hi, C_sigma lo into tensor memory: plane v at columns 64 v, lane m, column c = the bf16 pair
    // (k = 2c, 2c + 1) of row m
#pragma unroll 1
    for (int v = 0; v < 4; v++) {
        constexpr int kw = 64 / kGroups;  // bf16 pairs of the plane's row per thread
        const uint32_t *src = reinterpret_cast<const uint32_t *>(a.c_planes + ((size_t)v * kN + L) * kN) + kw * g;
#pragma unroll
        for (int c0 = 0; c0 < kw; c0 += 8) {
            float r[8];
#pragma unroll
            for (int i = 0; i < 8; i++) r[i] = __uint_as_float(src[c0 + i]);
            tmem_st8(lane_addr + 64 * v + kw * g + c0, r);
        }
    }
    tmem_wait_st();
    uint32_t phase = 0u, pending = 0u;  // bit x: parity to wait for / commit outstanding, of plane x's barrier
    bool bad = false;
    // waits for plane x's MMAs; a wait that runs out marks this thread bad and raises the fault flag
    auto wait_plane = [&](int x) {
        if (mbar_wait(&mbar[x], (phase >> x) & 1u, kWaitLimit)) {
            phase ^= 1u << x;
            pending &= ~(1u << x);
        } else {
            bad = true;
            *a.fault = 1;
        }
        fence_after_sync();
    };
    // publishes this thread's B-operand writes and tensor-memory reads; false (for every thread) when any thread is bad
    auto publish = [&]() -> bool {
        fence_proxy_async();
        fence_before_sync();
        const int any_bad = __syncthreads_or(bad ? 1 : 0);
        fence_after_sync();
        return any_bad == 0;
    };
    const float inv_n = 1.0f / (float)(kN * kN);
    for (int p = a.first + blockIdx.x; p < last; p += gridDim.x) {
        // ---- stage 1: B[n = r][k = c] = X.  Warp w takes rows kRowsPerWarp w .. + kRowsPerWarp - 1, each in two halves
        // of 64 columns; lane i the columns 2i, 2i + 1 of a half: one contiguous 512-byte segment of the object row and
        // of the probe row per warp and load, one 4-byte bf16 pair per plane and lane per store.
        {
            const int rr = a.scan.rr[p], cc = a.scan.cc[p], cls = a.scan.cls[p];
            const int OC = a.object_columns;
            const int row0 = kRowsPerWarp * warp;  // the warp's first patch row
            const float2 *S = a.shifted + (size_t)cls * (kN * kN) + row0 * kN + 2 * lane;
            // patch rows row0 .. row0 + kRowsPerWarp - 1 are object rows y0 .. (wrapped), y0 = rr + row0, or
            // rr + row0 - 128 past the centre row (a warp's rows never straddle it)
            const int y0 = rr + (row0 < kN / 2 ? row0 : row0 - kN);
            // the patch row is the object row segment [cc - 64, cc + 64) (its columns 64..127, then 0..63): one
            // aligned float4 per lane and half when it does not wrap and starts on an even complex
            if (cc >= kN / 2 && cc + kN / 2 <= OC && ((cc | OC) & 1) == 0) {
#pragma unroll
                for (int b0 = 0; b0 < kRowsPerWarp; b0 += kBatch) {  // kBatch rows, both halves: 4 kBatch loads in flight
                    float4 sv[2 * kBatch], ov[2 * kBatch];
#pragma unroll
                    for (int i = 0; i < kBatch; i++) {
                        const float2 *orow = a.object + (size_t)wrap_once(y0 + b0 + i, a.object_rows) * OC + cc + 2 * lane;
                        sv[2 * i] = __ldg(reinterpret_cast<const float4 *>(S + (b0 + i) * kN));
                        sv[2 * i + 1] = __ldg(reinterpret_cast<const float4 *>(S + (b0 + i) * kN + kN / 2));
                        ov[2 * i] = __ldg(reinterpret_cast<const float4 *>(orow));
                        ov[2 * i + 1] = __ldg(reinterpret_cast<const float4 *>(orow - kN / 2));
                    }
#pragma unroll
                    for (int u = 0; u < 2 * kBatch; u++) {
                        const float4 sp = sv[u], o = ov[u];
                        uint32_t rh, rl, ih, il;
                        split_bf16x2(sp.x * o.x - sp.y * o.y, sp.z * o.z - sp.w * o.w, rh, rl);
                        split_bf16x2(sp.x * o.y + sp.y * o.x, sp.z * o.w + sp.w * o.z, ih, il);
                        // row row0 + b0 + u/2, columns 64 (u & 1) + 2 lane
                        const uint32_t off = kmajor_offset(row0 + b0 + (u >> 1), 64 * (u & 1) + 2 * lane);
                        *reinterpret_cast<uint32_t *>(planes + (kReHi + 0) * kPlaneBytes + off) = rh;
                        *reinterpret_cast<uint32_t *>(planes + (kReHi + 1) * kPlaneBytes + off) = rl;
                        *reinterpret_cast<uint32_t *>(planes + (kImHi + 0) * kPlaneBytes + off) = ih;
                        *reinterpret_cast<uint32_t *>(planes + (kImHi + 1) * kPlaneBytes + off) = il;
                    }
                }
            } else {
                // near the object's edge (or an odd row length): complex by complex, each column wrapped
#pragma unroll 1
                for (int u = 0; u < 2 * kRowsPerWarp; u++) {
                    const int i = u >> 1, c = 64 * (u & 1) + 2 * lane;
                    const float2 *orow = a.object + (size_t)wrap_once(y0 + i, a.object_rows) * OC;
                    const int x = cc + (c < kN / 2 ? c : c - kN);
                    const float4 sp = __ldg(reinterpret_cast<const float4 *>(S + i * kN + 64 * (u & 1)));
                    const float2 o0 = __ldg(orow + wrap_once(x, OC)), o1 = __ldg(orow + wrap_once(x + 1, OC));
                    uint32_t rh, rl, ih, il;
                    split_bf16x2(sp.x * o0.x - sp.y * o0.y, sp.z * o1.x - sp.w * o1.y, rh, rl);
                    split_bf16x2(sp.x * o0.y + sp.y * o0.x, sp.z * o1.y + sp.w * o1.x, ih, il);
                    const uint32_t off = kmajor_offset(row0 + i, c);
                    *reinterpret_cast<uint32_t *>(planes + (kReHi + 0) * kPlaneBytes + off) = rh;
                    *reinterpret_cast<uint32_t *>(planes + (kReHi + 1) * kPlaneBytes + off) = rl;
                    *reinterpret_cast<uint32_t *>(planes + (kImHi + 0) * kPlaneBytes + off) = ih;
                    *reinterpret_cast<uint32_t *>(planes + (kImHi + 1) * kPlaneBytes + off) = il;
                }
            }
        }
        if (!publish()) break;
        if (tid == 0) {
            issue_plane(tmem, kCNat, kSlotRe, smem + kReHi * kPlaneBytes, kIdescK);
            mma_commit(&mbar[0]);
            issue_plane(tmem, kCNat, kSlotIm, smem + kImHi * kPlaneBytes, kIdescK);
            mma_commit(&mbar[1]);
        }
        pending = 3u;
        // ---- stage 2: B[n = raw c][k = r] = D1, each plane as soon as its stage-1 product is done
        wait_plane(0);
        readout_kmajor(lane_addr + kSlotRe + kCols * g, planes, kReHi, L, kCols * g);
        if (!publish()) break;
        if (tid == 0) {
            issue_plane(tmem, kCNat, kSlotRe, smem + kReHi * kPlaneBytes, kIdescK);
            mma_commit(&mbar[0]);
        }
        pending |= 1u;
        wait_plane(1);
        readout_kmajor(lane_addr + kSlotIm + kCols * g, planes, kImHi, L, kCols * g);
        if (!publish()) break;
        if (tid == 0) {
            issue_plane(tmem, kCNat, kSlotIm, smem + kImHi * kPlaneBytes, kIdescK);
            mma_commit(&mbar[1]);
        }
        pending |= 2u;
        // ---- projection on F (rows kr = j, mirror(j); this thread's 16 columns kc); stage 3: B = F', MN-major
        wait_plane(0);
        wait_plane(1);
        if (mbar_wait(&amp_bar, amp_phase, kWaitLimit)) {
            amp_phase ^= 1u;
            amp_pending = false;
        } else {
            bad = true;
            *a.fault = 1;
        }
        {
            // the squared residual of this thread's 32 frequencies in FP32 (two packed lanes), then in FP64 over the
            // threads, warps and positions, as the reference's Float path sums a pattern in Float and the patterns in
            // Double (PtychographySingle.swift:157-172)
            float2 errv = make_float2(0.f, 0.f);
            const float2 inv_n2 = make_float2(inv_n, inv_n), minus_one = make_float2(-1.f, -1.f);
#pragma unroll 1
            for (int u = 0; u < kSub; u++) {
                float4 am4[4];
#pragma unroll
                for (int e = 0; e < 4; e++) am4[e] = amp_smem[(4 * u + e) * kThreads + tid];
                float fr[2][8], fi[2][8];
                combined_block<false>(lane_addr, g, u, j, h, fr, fi);
#pragma unroll
                for (int side = 0; side < 2; side++) {
#pragma unroll
                    for (int e = 0; e < 8; e += 2) {  // two frequencies per packed instruction
                        const float4 av = am4[2 * side + (e >> 2)];
                        const float2 am = (e & 2) ? make_float2(av.z, av.w) : make_float2(av.x, av.y);
                        const float2 re = make_float2(fr[side][e], fr[side][e + 1]);
                        const float2 im = make_float2(fi[side][e], fi[side][e + 1]);
                        // |F| and A / |F| through one reciprocal square root; F = 0 takes the amplitude itself
                        const float2 m2 = pfma(re, re, pmul(im, im));
                        const bool nz0 = m2.x > 0.f, nz1 = m2.y > 0.f;
                        const float2 inv = make_float2(rsqrtf(m2.x), rsqrtf(m2.y));
                        const float2 mag = pmul(m2, inv);
                        const float2 miss = psub(am, make_float2(nz0 ? mag.x : 0.f, nz1 ? mag.y : 0.f));
                        errv = pfma(miss, miss, errv);
                        const float2 sc = pmul(pfma(am, inv, minus_one), inv_n2);
                        const float2 nr = pmul(re, sc), ni = pmul(im, sc), zr = pmul(am, inv_n2);
                        fr[side][e] = nz0 ? nr.x : zr.x;
                        fr[side][e + 1] = nz1 ? nr.y : zr.y;
                        fi[side][e] = nz0 ? ni.x : 0.f;
                        fi[side][e + 1] = nz1 ? ni.y : 0.f;
                    }
                    const uint32_t off = mnmajor_offset(side ? mirror(j) : j, kCols * g + (kCols / 2) * h + 8 * u);
                    store_split8(planes, kReHi, off, fr[side]);
                    store_split8(planes, kImHi, off, fi[side]);
                }
            }
            double err = (double)errv.x + (double)errv.y;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) err += __shfl_down_sync(0xffffffffu, err, o);
            if (lane == 0) a.error[(size_t)p * (kThreads / 32) + warp] = err;
        }
        if (!publish()) break;
        if (tid == 0) {
            issue_plane(tmem, kCNat, kSlotRe, smem + kReHi * kPlaneBytes, kIdescMN);
            mma_commit(&mbar[0]);
            issue_plane(tmem, kCNat, kSlotIm, smem + kImHi * kPlaneBytes, kIdescMN);
            mma_commit(&mbar[1]);
            // every thread has read this position's amplitudes: fetch the next one's behind stages 3 to 2
            if (p + (int)gridDim.x < last)
                bulk_load(amp_smem, a.amplitudes + (size_t)(p + gridDim.x) * (kN * kN), kN * kN * 4, &amp_bar);
        }
        amp_pending = p + (int)gridDim.x < last;
        pending = 3u;
        // ---- stage 4: B[n = raw r][k = pos] = D3, contracted with C_sigma
        wait_plane(0);
        readout_kmajor(lane_addr + kSlotRe + kCols * g, planes, kReHi, L, kCols * g);
        if (!publish()) break;
        if (tid == 0) {
            issue_plane(tmem, kCSigma, kSlotRe, smem + kReHi * kPlaneBytes, kIdescK);
            mma_commit(&mbar[0]);
        }
        pending |= 1u;
        wait_plane(1);
        readout_kmajor(lane_addr + kSlotIm + kCols * g, planes, kImHi, L, kCols * g);
        if (!publish()) break;
        if (tid == 0) {
            issue_plane(tmem, kCSigma, kSlotIm, smem + kImHi * kPlaneBytes, kIdescK);
            mma_commit(&mbar[1]);
        }
        pending |= 2u;
        // ---- dpsi[r][c]: columns c = j, mirror(j) of this lane pair, rows r = J, mirror(J)
        wait_plane(0);
        wait_plane(1);
        {
            float2 *out = a.dpsi + (size_t)(p - a.dpsi_first) * (kN * kN);
#pragma unroll 1
            for (int u = 0; u < kSub; u++) {
                float dr[2][8], di[2][8];
                combined_block<true>(lane_addr, g, u, j, h, dr, di);
#pragma unroll
                for (int side = 0; side < 2; side++) {
                    const int c = side ? mirror(j) : j;
#pragma unroll
                    for (int e = 0; e < 8; e++) {
                        const int J = column_of(g, h, u, e & 3);
                        const int r = (e >> 2) ? mirror(J) : J;
                        out[r * kN + c] = make_float2(dr[side][e], di[side][e]);
                    }
                }
            }
        }
        // the next position's stage 1 overwrites the B planes (its MMAs are issued after the next publish)
    }
    fence_before_sync();
    if (__syncthreads_or(bad ? 1 : 0)) {
        // a wait ran out: give the tensor core a bounded chance to drain before the columns are freed
        for (int x = 0; x < 2; x++)
            if ((pending >> x) & 1u) mbar_wait(&mbar[x], (phase >> x) & 1u, kWaitLimit);
        if (amp_pending) mbar_wait(&amp_bar, amp_phase, kWaitLimit);  // no copy may land after the CTA has gone
    }
    fence_after_sync();
    if (warp == 0) tmem_dealloc(tmem, 512);
}

// [position][row][column] -> [position][e4][thread][4]: thread T's float4 e4 = 4 u + 2 side + s holds the amplitudes of
// row (side ? mirror(j) : j), columns (s ? mirror(J) : J), J = column_of(g, h, u, i), i = 0..3, for T's lane pair j,
// parity h and column group g.
__global__ void permute_bf16_amplitudes_kernel(const float *in, float *out, long long positions) {
    const long long idx = (long long)blockIdx.x * 256 + threadIdx.x;
    if (idx >= positions * kN * kN) return;
    const long long p = idx / (kN * kN);
    const int rem = (int)(idx - p * kN * kN);
    const int i = rem & 3, T = (rem >> 2) & (kThreads - 1), e4 = (rem >> 2) / kThreads;
    const int u = e4 >> 2, side = (e4 >> 1) & 1, s = e4 & 1;
    const int w = T >> 5, L = 32 * (w & 3) + (T & 31), g = w >> 2;
    const int jj = L >> 1, h = L & 1;
    const int J = column_of(g, h, u, i);
    const int kc = s ? mirror(J) : J, kr = side ? mirror(jj) : jj;
    out[idx] = in[p * kN * kN + kr * kN + kc];
}

size_t bf16_smem() { return 4 * (size_t)kPlaneBytes + (size_t)kN * kN * sizeof(float); }

}  // namespace

bool bf16_applicable(int rows, int columns) { return rows == kN && columns == kN; }
int bf16_partials_per_position() { return kThreads / 32; }

// Stage 3's contraction position pos = kCols g + (kCols / 2) h + 8 u + 4 s + i holds the frequency
// s ? mirror(J) : J, J = column_of(g, h, u, i): the order in which a thread stores its projected values.
int bf16_sigma(int pos) {
    const int g = pos / kCols, h = (pos % kCols) / (kCols / 2), r = pos % (kCols / 2);
    const int u = r >> 3, s = (r >> 2) & 1, i = r & 3;
    const int J = column_of(g, h, u, i);
    return s ? mirror(J) : J;
}

cudaError_t configure_bf16() {
    int device = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    if ((size_t)optin < bf16_smem() + 1024) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(bf16_position_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bf16_smem());
}

cudaError_t launch_bf16(const Bf16Args &a, int ctas, cudaStream_t s) {
    if (a.count <= 0) return cudaSuccess;
    const int grid = a.count < ctas ? a.count : ctas;
    bf16_position_kernel<<<grid, kThreads, bf16_smem(), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_permute_bf16_amplitudes(const float *in, float *out, long long positions, cudaStream_t s) {
    const long long total = positions * kN * kN;
    permute_bf16_amplitudes_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(in, out, positions);
    return cudaGetLastError();
}

}  // namespace cubo
