// Device parse of the reference's adjacency text into the resident CSR (declarations in ingest.cuh).
//
// Semantics (the reference's load_graph, src/phase1/init.cpp:15-100, as the host loader adjtext.cpp
// restates them): the body is every newline-terminated line after the header; line v lists the neighbours
// of vertex v.  fast_atoi tokenisation: a token starts at the first byte of a non-empty line and at every
// digit that follows a non-digit; its value is its run of digits (empty: 0).  A NUL byte ends the parse of
// its line.  The raw degree is the token count; the CSR row is the sorted, de-duplicated token list
// (src/phase1/partition.cpp:227-262, self-loops kept).  An id >= V is rejected.
//
// Text passes are tiled: a block reads 16 KiB as 4 steps of 256 coalesced 16-byte loads, classifies the
// 16 bytes of a load with byte-SIMD compares into newline / digit / NUL bit masks, and emits tokens in
// text order from a block scan of per-thread counts plus the tile's prefix (count pass -> scan -> emit
// pass).  Rows that are not strictly increasing (only in hand-written input: the reference's converter
// writes sorted rows) are sorted on the device, by length class, then de-duplicated by a token scan.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "device_state.cuh"
#include "ingest.cuh"

namespace dmolp {
namespace ingest {
namespace {

constexpr uint32_t kFirst = 0x80000000u;  // token flag: first token of its line
constexpr uint32_t kVal = 0x7fffffffu;
constexpr int kSmallRow = 32;             // unsorted rows up to this length: one thread sorts
constexpr int kMidRow = 4096;             // ... up to this length: one block, in shared memory
constexpr int kNW = kTxtThreads / 32;

struct Scal {
    unsigned long long nul;         // NUL bytes in the body
    unsigned long long violations;  // tokens not above their predecessor in the same line
    unsigned long long maxdeg, maxraw;
    int bad_id;                     // some token >= V
    int nlist[3];                   // unsorted rows per length class
};

// Byte tests on a 32-bit word, one flag per byte in bit 7 of that byte.  Exact for every byte value: the
// additions work on 7-bit fields, so no carry crosses into the next byte.
__device__ __forceinline__ uint32_t zero_bytes(uint32_t w) { return ~(((w & 0x7f7f7f7fu) + 0x7f7f7f7fu) | w) & 0x80808080u; }
__device__ __forceinline__ uint32_t digit_bytes(uint32_t w) {  // '0'..'9'
    const uint32_t lo = w & 0x7f7f7f7fu;
    return (lo + 0x50505050u) & ~(lo + 0x46464646u) & ~w & 0x80808080u;
}
// bit-7 byte flags -> 4-bit mask (byte 0 -> bit 0)
__device__ __forceinline__ uint32_t byte_bits(uint32_t m) { return (m * 0x00204081u) >> 28; }

struct Chunk {
    uint32_t nl, zero, dig, body, ts;  // 16-bit masks over the chunk's bytes; ts = token starts
    uint32_t prev_nl;                  // (nl << 1) | previous byte is a newline
};

// Classify the 16 bytes at `pos` (16-aligned).  All 32 lanes must call it (the previous byte comes from
// the neighbouring lane).
__device__ __forceinline__ Chunk chunk_at(const uint8_t *__restrict__ txt, int64_t pos, int64_t body0, int64_t body1,
                                         uint4 *raw = nullptr) {
    const uint4 q = __ldg(reinterpret_cast<const uint4 *>(txt + pos));
    if (raw) *raw = q;
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
    Chunk c;
    c.nl = c.zero = c.dig = 0;
    uint32_t anyz = 0;
    uint32_t zw[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        c.nl |= byte_bits(zero_bytes(w[i] ^ 0x0a0a0a0au)) << (4 * i);
        c.dig |= byte_bits(digit_bytes(w[i])) << (4 * i);
        zw[i] = zero_bytes(w[i]);
        anyz |= zw[i];
    }
    if (anyz) {  // NUL bytes: the tile padding, or a NUL in the text
#pragma unroll
        for (int i = 0; i < 4; ++i) c.zero |= byte_bits(zw[i]) << (4 * i);
    }
    const int lane = threadIdx.x & 31;
    uint32_t pb = __shfl_up_sync(DMOLP_FULL_MASK, q.w >> 24, 1);
    if (lane == 0) pb = pos > 0 ? txt[pos - 1] : 0u;
    const uint32_t pnl = pb == '\n', pdig = pb - '0' <= 9u;
    const int64_t lo = body0 - pos, hi = body1 - pos;
    const uint32_t below = lo <= 0 ? 0u : (lo >= 16 ? 0xffffu : (1u << lo) - 1);
    const uint32_t upto = hi <= 0 ? 0u : (hi >= 16 ? 0xffffu : (1u << hi) - 1);
    c.body = upto & ~below;
    c.prev_nl = ((c.nl << 1) | pnl) & 0xffffu;
    const uint32_t prev_dig = ((c.dig << 1) | pdig) & 0xffffu;
    c.ts = c.body & ~c.nl & ~c.zero & (c.prev_nl | (c.dig & ~prev_dig));
    return c;
}

// Value of a run of 1..8 ASCII digits held little-endian in v (first digit in the lowest byte): left-pad to
// eight digits with '0', then combine digit pairs, quads and halves with three multiplications (Lemire's
// eight-digit SWAR parse, "Faster integer parsing", 2021).
__device__ __forceinline__ uint32_t parse_digits8(uint64_t v, int n) {
    if (n < 8) v = (v << (8 * (8 - n))) | (0x3030303030303030ull >> (8 * n));
    v = ((v & 0x0f0f0f0f0f0f0f0full) * 2561) >> 8;
    v = ((v & 0x00ff00ff00ff00ffull) * 6553601) >> 16;
    return (uint32_t)(((v & 0x0000ffff0000ffffull) * 42949672960001ull) >> 32);
}

// Exclusive block scan of a 32-bit value (packed counters whose block totals cannot carry).
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *total, uint32_t *s_w) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(DMOLP_FULL_MASK, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        uint32_t x = lane < kNW ? s_w[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(DMOLP_FULL_MASK, x, o);
            if (lane >= o) x += y;
        }
        if (lane < kNW) s_w[lane] = x;
    }
    __syncthreads();
    const uint32_t before = wid ? s_w[wid - 1] : 0u;
    *total = s_w[kNW - 1];
    __syncthreads();  // s_w is reused by the next call
    return before + incl - v;
}

__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t *s_w) {
    uint32_t t;
    block_excl_scan(v, &t, s_w);
    return t;
}

// ---- text passes ----

__global__ void __launch_bounds__(kTxtThreads) k_txt_count(const uint8_t *__restrict__ txt, int64_t body0,
                                                           int64_t body1, uint32_t *__restrict__ tcnt, Scal *sc) {
    __shared__ uint32_t s_w[kNW];
    const int64_t tile = blockIdx.x;
    uint32_t nl = 0, tk = 0, nz = 0;
#pragma unroll
    for (int s = 0; s < kTxtSteps; ++s) {
        const int64_t pos = tile * kTileBytes + (int64_t)(s * kTxtThreads + threadIdx.x) * kChunkBytes;
        const Chunk c = chunk_at(txt, pos, body0, body1);
        nl += __popc(c.nl & c.body);
        tk += __popc(c.ts);
        nz += __popc(c.zero & c.body);
    }
    // tile totals are at most 16 Ki each: pack two per word
    const uint32_t nlt = block_sum(nl | (tk << 16), s_w);
    const uint32_t nzt = block_sum(nz, s_w);
    if (threadIdx.x == 0) {
        tcnt[2 * tile] = nlt & 0xffffu;
        tcnt[2 * tile + 1] = nlt >> 16;
        if (nzt) atomicAdd(&sc->nul, (unsigned long long)nzt);
    }
}

// A NUL ends the parse of its line: zero every byte from each NUL up to the next NUL or newline, so that
// no token starts after the first NUL of a line.  Writers only ever store zeros below the line's newline,
// so overlapping walks are harmless.
__global__ void k_txt_nulfill(uint8_t *txt, int64_t body0, int64_t body1) {
    const int64_t c0 = body0 / 16, c1 = (body1 + 15) / 16;
    for (int64_t ci = c0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; ci < c1;
         ci += (int64_t)gridDim.x * blockDim.x) {
        for (int j = 0; j < 16; ++j) {
            const int64_t p = ci * 16 + j;
            if (p < body0 || p >= body1 || txt[p] != 0) continue;
            for (int64_t q = p + 1; q < body1; ++q) {
                const uint8_t b = ((volatile uint8_t *)txt)[q];
                if (b == '\n' || b == 0) break;
                ((volatile uint8_t *)txt)[q] = 0;
            }
        }
    }
}

// Exclusive prefix over n records of NC 32-bit counters: out[i*NC+c] = sum_{j<i} cnt[j*NC+c],
// out[n*NC+c] = total.  One block; each thread owns a contiguous range of records.
template <int NC>
__global__ void __launch_bounds__(1024) k_scan(const uint32_t *__restrict__ cnt, int64_t n, int64_t *__restrict__ out) {
    __shared__ long long s_w[32][NC];
    const int T = blockDim.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int64_t per = (n + T - 1) / T;
    const int64_t a = std::min<int64_t>(n, tid * per), z = std::min<int64_t>(n, a + per);
    long long s[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) s[c] = 0;
    for (int64_t i = a; i < z; ++i)
#pragma unroll
        for (int c = 0; c < NC; ++c) s[c] += cnt[i * NC + c];
    long long incl[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        incl[c] = s[c];
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(DMOLP_FULL_MASK, incl[c], o);
            if (lane >= o) incl[c] += y;
        }
        if (lane == 31) s_w[wid][c] = incl[c];
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = T / 32;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            long long x = lane < nw ? s_w[lane][c] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const long long y = __shfl_up_sync(DMOLP_FULL_MASK, x, o);
                if (lane >= o) x += y;
            }
            if (lane < nw) s_w[lane][c] = x;
        }
    }
    __syncthreads();
    long long run[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) run[c] = (wid ? s_w[wid - 1][c] : 0) + incl[c] - s[c];
    for (int64_t i = a; i < z; ++i)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            out[i * NC + c] = run[c];
            run[c] += cnt[i * NC + c];
        }
    if (tid == T - 1)
#pragma unroll
        for (int c = 0; c < NC; ++c) out[n * NC + c] = run[c];
}

// Tokens in text order: value (bit 31 = first token of its line); end_tok[l] = tokens before line l's
// newline.  Per step a warp owns a 512-byte window: the lanes classify their 16 bytes, stage them in
// shared memory with the window's token starts, then parse the window's tokens round-robin (lane i takes
// tokens i, i+32, ...), so the digit loops are balanced across the warp and the stores are coalesced.
// Values are parsed with saturation at 2^31, so any id >= V is caught.
constexpr int kWin = 32 * kChunkBytes;  // bytes of a warp's window
constexpr int kLook = 32;               // look-ahead staged past the window

__global__ void __launch_bounds__(kTxtThreads) k_txt_emit(const uint8_t *__restrict__ txt, int64_t body0,
                                                          int64_t body1, int64_t nv, const int64_t *__restrict__ toff,
                                                          uint32_t *__restrict__ tok, int64_t *__restrict__ end_tok,
                                                          Scal *sc) {
    __shared__ uint32_t s_w[kNW];
    __shared__ __align__(16) uint8_t s_txt[kNW][kWin + kLook];
    __shared__ uint16_t s_pos[kNW][kWin];  // window offset of each token start; bit 15 = first of its line
    const int64_t tile = blockIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint8_t *wt = s_txt[wid];
    uint16_t *wp = s_pos[wid];
    int64_t lbase = toff[2 * tile], tbase = toff[2 * tile + 1];
    int bad = 0;
#pragma unroll 1
    for (int s = 0; s < kTxtSteps; ++s) {
        const int64_t pos = tile * kTileBytes + (int64_t)(s * kTxtThreads + threadIdx.x) * kChunkBytes;
        uint4 q;
        const Chunk c = chunk_at(txt, pos, body0, body1, &q);
        reinterpret_cast<uint4 *>(wt)[lane] = q;
        if (lane < kLook / 16)  // the bytes after the window, for digit runs that cross its end
            reinterpret_cast<uint4 *>(wt + kWin)[lane] =
                __ldg(reinterpret_cast<const uint4 *>(txt + pos - lane * kChunkBytes + kWin) + lane);
        const uint32_t nlm = c.nl & c.body;
        const uint32_t ntk = (uint32_t)__popc(c.ts);
        uint32_t tot;
        const uint32_t ex = block_excl_scan((uint32_t)__popc(nlm) << 16 | ntk, &tot, s_w);
        const int64_t t0 = tbase + (ex & 0xffffu);  // this lane's first token
        int64_t l = lbase + (ex >> 16);
        const uint32_t wex = __shfl_sync(DMOLP_FULL_MASK, ex & 0xffffu, 0);
        const int o = (int)((ex & 0xffffu) - wex);  // offset of this lane's tokens in the window's list
        const int wtot = __shfl_sync(DMOLP_FULL_MASK, o + (int)ntk, 31);
        uint32_t m = c.ts;
        for (int k = 0; m; ++k) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            wp[o + k] = (uint16_t)(lane * kChunkBytes + j) | (((c.prev_nl >> j) & 1u) ? 0x8000u : 0u);
        }
        for (uint32_t n = nlm; n; n &= n - 1) {
            const int j = __ffs(n) - 1;
            end_tok[l++] = t0 + __popc(c.ts & ((1u << j) - 1));
        }
        __syncwarp();
        const int64_t tw = t0 - o;  // the window's first token
        for (int i = lane; i < wtot; i += 32) {
            const uint32_t e = wp[i];
            const int x0 = (int)(e & 0x7fffu);
            // the 8 bytes from the token start, out of three aligned words of the staged window
            const uint32_t *w32 = reinterpret_cast<const uint32_t *>(wt) + (x0 >> 2);
            const uint32_t a0 = w32[0], a1 = w32[1], a2 = w32[2], a3 = w32[3];
            const uint32_t sh = 8u * (x0 & 3);
            const uint32_t lo = __funnelshift_r(a0, a1, sh), hi = __funnelshift_r(a1, a2, sh);
            const uint32_t nx = __funnelshift_r(a2, a3, sh);  // bytes 8..11 of the token
            const uint32_t dm = byte_bits(digit_bytes(lo)) | byte_bits(digit_bytes(hi)) << 4 |
                                byte_bits(digit_bytes(nx)) << 8;
            const int n = __ffs(~dm) - 1;  // leading digits (0..12)
            uint32_t x;
            if (n <= 8) {
                x = n ? parse_digits8((uint64_t)hi << 32 | lo, n) : 0u;
            } else {  // nine digits or more (ids >= 10^8, or leading zeros): digit by digit
                int64_t g = pos - lane * kChunkBytes + x0;
                x = 0;
                for (uint32_t b = txt[g]; b - '0' <= 9u; b = txt[++g]) x = x > 214748364u ? 0x80000000u : x * 10 + (b - '0');
            }
            if ((int64_t)x >= nv) bad = 1;
            tok[tw + i] = (x & kVal) | ((e & 0x8000u) ? kFirst : 0u);
        }
        lbase += tot >> 16;
        tbase += tot & 0xffffu;
        __syncwarp();
    }
    if (bad) atomicOr(&sc->bad_id, 1);
}

// ---- row order ----

__device__ __forceinline__ int64_t row_of(const int64_t *__restrict__ end_tok, int64_t nv, int64_t t) {
    int64_t lo = 0, hi = nv;  // first line whose newline comes after token t
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (end_tok[mid] > t) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

__global__ void k_tok_check(const uint32_t *__restrict__ tok, int64_t ntok, const int64_t *__restrict__ end_tok,
                            int64_t nv, uint8_t *__restrict__ badrow, Scal *sc) {
    unsigned long long nbad = 0;
    for (int64_t t = 1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ntok; t += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t cur = tok[t];
        if (cur & kFirst) continue;
        if ((cur & kVal) <= (tok[t - 1] & kVal)) {
            ++nbad;
            badrow[row_of(end_tok, nv, t)] = 1;
        }
    }
    nbad = warp_sum_u64(nbad);
    if ((threadIdx.x & 31) == 0 && nbad) atomicAdd(&sc->violations, nbad);
}

__global__ void k_rows_classify(const int64_t *__restrict__ end_tok, int64_t nv, const uint8_t *__restrict__ badrow,
                                int32_t *__restrict__ lists, Scal *sc) {
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < nv; l += (int64_t)gridDim.x * blockDim.x) {
        if (!badrow[l]) continue;
        const int64_t len = end_tok[l] - (l ? end_tok[l - 1] : 0);
        const int cls = len <= kSmallRow ? 0 : (len <= kMidRow ? 1 : 2);
        lists[cls * nv + atomicAdd(&sc->nlist[cls], 1)] = (int32_t)l;
    }
}

__device__ __forceinline__ void row_bounds(const int64_t *end_tok, int64_t l, int64_t *s, int64_t *e) {
    *s = l ? end_tok[l - 1] : 0;
    *e = end_tok[l];
}

__global__ void k_sort_small(uint32_t *__restrict__ tok, const int64_t *__restrict__ end_tok,
                             const int32_t *__restrict__ list, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t s, e;
    row_bounds(end_tok, list[i], &s, &e);
    const int len = (int)(e - s);
    uint32_t a[kSmallRow];
    for (int j = 0; j < len; ++j) {
        const uint32_t x = tok[s + j] & kVal;
        int q = j;
        while (q > 0 && a[q - 1] > x) {
            a[q] = a[q - 1];
            --q;
        }
        a[q] = x;
    }
    for (int j = 0; j < len; ++j) tok[s + j] = a[j] | (j == 0 ? kFirst : 0u);
}

// In-place bitonic sort of a[0..P) (P a power of two) by all threads of the block.
__device__ __forceinline__ void bitonic(uint32_t *a, int P) {
    for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += blockDim.x) {
                const int x = i ^ j;
                if (x > i) {
                    const uint32_t u = a[i], v = a[x];
                    if ((u > v) == ((i & k) == 0)) {
                        a[i] = v;
                        a[x] = u;
                    }
                }
            }
            __syncthreads();
        }
}

__global__ void __launch_bounds__(512) k_sort_mid(uint32_t *__restrict__ tok, const int64_t *__restrict__ end_tok,
                                                  const int32_t *__restrict__ list) {
    __shared__ uint32_t a[kMidRow];
    int64_t s, e;
    row_bounds(end_tok, list[blockIdx.x], &s, &e);
    const int len = (int)(e - s);
    int P = 2;
    while (P < len) P <<= 1;
    for (int i = threadIdx.x; i < P; i += blockDim.x) a[i] = i < len ? (tok[s + i] & kVal) : 0xffffffffu;
    __syncthreads();
    bitonic(a, P);
    for (int i = threadIdx.x; i < len; i += blockDim.x) tok[s + i] = a[i] | (i == 0 ? kFirst : 0u);
}

// Rows above kMidRow tokens: sort kMidRow-token chunks in shared memory, then merge pairs of runs in
// global memory (tok <-> tmp), the block's threads splitting each merge's output along the merge path.
__global__ void __launch_bounds__(1024) k_sort_big(uint32_t *__restrict__ tok, uint32_t *__restrict__ tmp,
                                                   const int64_t *__restrict__ end_tok, const int32_t *__restrict__ list) {
    __shared__ uint32_t a[kMidRow];
    int64_t s, e;
    row_bounds(end_tok, list[blockIdx.x], &s, &e);
    const int64_t len = e - s;
    uint32_t *src = tok + s, *dst = tmp + s;
    for (int64_t c0 = 0; c0 < len; c0 += kMidRow) {
        const int n = (int)std::min<int64_t>(kMidRow, len - c0);
        for (int i = threadIdx.x; i < kMidRow; i += blockDim.x) a[i] = i < n ? (src[c0 + i] & kVal) : 0xffffffffu;
        __syncthreads();
        bitonic(a, kMidRow);
        for (int i = threadIdx.x; i < n; i += blockDim.x) src[c0 + i] = a[i];
        __syncthreads();
    }
    for (int64_t w = kMidRow; w < len; w <<= 1) {
        for (int64_t a0 = 0; a0 < len; a0 += 2 * w) {
            const int64_t na = std::min<int64_t>(w, len - a0), nb = std::min<int64_t>(w, len - a0 - na);
            const uint32_t *X = src + a0, *Y = src + a0 + na;
            uint32_t *O = dst + a0;
            const int64_t n = na + nb, per = (n + blockDim.x - 1) / blockDim.x;
            const int64_t d0 = std::min<int64_t>(n, threadIdx.x * per), d1 = std::min<int64_t>(n, d0 + per);
            if (d0 >= d1) continue;
            int64_t lo = std::max<int64_t>(0, d0 - nb), hi = std::min<int64_t>(d0, na);
            while (lo < hi) {  // elements of X among the first d0 outputs (ties: X first)
                const int64_t mid = (lo + hi) >> 1;
                if (X[mid] <= Y[d0 - 1 - mid]) lo = mid + 1;
                else hi = mid;
            }
            int64_t i = lo, j = d0 - lo;
            for (int64_t d = d0; d < d1; ++d) {
                if (j >= nb || (i < na && X[i] <= Y[j])) O[d] = X[i++];
                else O[d] = Y[j++];
            }
        }
        __syncthreads();
        uint32_t *t = src;
        src = dst;
        dst = t;
    }
    uint32_t *row = tok + s;
    for (int64_t i = threadIdx.x; i < len; i += blockDim.x) row[i] = src[i] | (i == 0 ? kFirst : 0u);
}

// ---- de-duplication: keep the first token of each line and every token unlike its predecessor ----

__device__ __forceinline__ bool kept(const uint32_t *tok, int64_t t) {
    const uint32_t x = tok[t];
    return (x & kFirst) || (x & kVal) != (tok[t - 1] & kVal);
}

__global__ void __launch_bounds__(kTxtThreads) k_keep_count(const uint32_t *__restrict__ tok, int64_t ntok,
                                                            uint32_t *__restrict__ tcnt) {
    __shared__ uint32_t s_w[kNW];
    uint32_t n = 0;
    for (int i = threadIdx.x; i < kTokTile; i += kTxtThreads) {
        const int64_t t = blockIdx.x * kTokTile + i;
        if (t < ntok) n += kept(tok, t);
    }
    const uint32_t tot = block_sum(n, s_w);
    if (threadIdx.x == 0) tcnt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kTxtThreads) k_keep_pos(const uint32_t *__restrict__ tok, int64_t ntok,
                                                          const int64_t *__restrict__ toff, int64_t *__restrict__ keptpos) {
    __shared__ uint32_t s_w[kNW];
    int64_t base = toff[blockIdx.x];
    for (int i0 = 0; i0 < kTokTile; i0 += kTxtThreads) {
        const int64_t t = blockIdx.x * kTokTile + i0 + threadIdx.x;
        const uint32_t k = t < ntok ? kept(tok, t) : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_scan(k, &tot, s_w);
        if (t < ntok) keptpos[t] = base + ex;
        base += tot;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) keptpos[ntok] = base;
}

// ---- per line: raw degree, CSR degree, classes ----

struct LineInfo {
    int64_t e_arc;  // arcs up to the end of the row (CSR offset of the next row)
    int64_t raw, deg;
    int cls;        // 0..2, or 3 for degree 0
};

__device__ __forceinline__ LineInfo line_info(const int64_t *__restrict__ end_tok, const int64_t *__restrict__ keptpos,
                                              int64_t l) {
    const int64_t s = l ? end_tok[l - 1] : 0, e = end_tok[l];
    LineInfo r;
    r.raw = e - s;
    if (keptpos) {
        r.e_arc = keptpos[e];
        r.deg = r.e_arc - keptpos[s];
    } else {
        r.e_arc = e;
        r.deg = r.raw;
    }
    r.cls = r.deg == 0 ? 3 : (r.deg <= kSmallDeg ? 0 : (r.deg <= kLargeDeg ? 1 : 2));
    return r;
}

__global__ void __launch_bounds__(kTxtThreads) k_lines_count(const int64_t *__restrict__ end_tok,
                                                             const int64_t *__restrict__ keptpos, int64_t nv,
                                                             uint32_t *__restrict__ lcnt, Scal *sc) {
    __shared__ uint32_t s_w[kNW];
    uint32_t cnt3 = 0;  // 10-bit fields
    unsigned long long md = 0, mr = 0;
    for (int s = 0; s < kLineSteps; ++s) {
        const int64_t l = blockIdx.x * kLineTile + s * kTxtThreads + threadIdx.x;
        if (l >= nv) break;
        const LineInfo r = line_info(end_tok, keptpos, l);
        if (r.cls < 3) cnt3 += 1u << (10 * r.cls);
        md = max(md, (unsigned long long)r.deg);
        mr = max(mr, (unsigned long long)r.raw);
    }
    // per-class totals of a tile reach 4096: sum the three fields separately
    const uint32_t c0 = block_sum(cnt3 & 1023u, s_w), c1 = block_sum((cnt3 >> 10) & 1023u, s_w),
                   c2 = block_sum(cnt3 >> 20, s_w);
    for (int o = 16; o > 0; o >>= 1) {
        md = max(md, __shfl_xor_sync(DMOLP_FULL_MASK, md, o));
        mr = max(mr, __shfl_xor_sync(DMOLP_FULL_MASK, mr, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (md) atomicMax(&sc->maxdeg, md);
        if (mr) atomicMax(&sc->maxraw, mr);
    }
    if (threadIdx.x == 0) {
        lcnt[3 * blockIdx.x] = c0;
        lcnt[3 * blockIdx.x + 1] = c1;
        lcnt[3 * blockIdx.x + 2] = c2;
    }
}

__global__ void __launch_bounds__(kTxtThreads) k_lines_emit(const int64_t *__restrict__ end_tok,
                                                            const int64_t *__restrict__ keptpos, int64_t nv,
                                                            const int64_t *__restrict__ loff, int64_t *__restrict__ off,
                                                            int32_t *__restrict__ raw, int32_t *b0, int32_t *b1,
                                                            int32_t *b2) {
    __shared__ uint32_t s_w[kNW];
    int64_t base[3] = {loff[3 * blockIdx.x], loff[3 * blockIdx.x + 1], loff[3 * blockIdx.x + 2]};
    if (blockIdx.x == 0 && threadIdx.x == 0) off[0] = 0;
    for (int s = 0; s < kLineSteps; ++s) {
        const int64_t l = blockIdx.x * kLineTile + s * kTxtThreads + threadIdx.x;
        if (blockIdx.x * kLineTile + s * kTxtThreads >= nv) break;  // uniform across the block
        LineInfo r;
        r.cls = 3;
        if (l < nv) {
            r = line_info(end_tok, keptpos, l);
            off[l + 1] = r.e_arc;
            raw[l] = (int32_t)r.raw;
        }
        // per-step class counts are at most 256: three 10-bit fields
        uint32_t tot;
        const uint32_t ex = block_excl_scan(r.cls < 3 ? 1u << (10 * r.cls) : 0u, &tot, s_w);
        if (r.cls < 3) {
            int32_t *b = r.cls == 0 ? b0 : (r.cls == 1 ? b1 : b2);
            b[base[r.cls] + ((ex >> (10 * r.cls)) & 1023u)] = (int32_t)l;
        }
        for (int c = 0; c < 3; ++c) base[c] += (tot >> (10 * c)) & 1023u;
    }
}

// ---- columns ----

__global__ void k_col_copy(const uint32_t *__restrict__ tok, int64_t ntok, int32_t *__restrict__ col) {
    const int64_t n4 = ntok / 4;
    const uint4 *src = reinterpret_cast<const uint4 *>(tok);
    int4 *dst = reinterpret_cast<int4 *>(col);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
        const uint4 q = __ldcs(src + i);
        __stcs(dst + i, make_int4((int)(q.x & kVal), (int)(q.y & kVal), (int)(q.z & kVal), (int)(q.w & kVal)));
    }
    for (int64_t t = n4 * 4 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ntok; t += (int64_t)gridDim.x * blockDim.x)
        col[t] = (int)(tok[t] & kVal);
}

__global__ void k_keep_compact(const uint32_t *__restrict__ tok, int64_t ntok, const int64_t *__restrict__ keptpos,
                               int32_t *__restrict__ col) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < ntok; t += (int64_t)gridDim.x * blockDim.x)
        if (kept(tok, t)) col[keptpos[t]] = (int)(tok[t] & kVal);
}

// ---- a binary CSR copied to the device as given (dmolp_graph_upload) ----

struct CsrScal {
    unsigned long long maxdeg, maxraw;
    unsigned long long violations;  // arcs not above their predecessor in the same row
    int bad;                        // 1: offsets, 2: an id outside [0, nv), 4: a negative raw degree
};

// Per vertex tile (kLineTile vertices): row bounds in [0, narcs] and non-decreasing, the degree classes'
// counts, the largest degree and raw degree, and a bit at the first arc of every non-empty row.
__global__ void __launch_bounds__(kTxtThreads) k_csr_rows(const int64_t *__restrict__ off,
                                                          const int32_t *__restrict__ raw, int64_t nv, int64_t narcs,
                                                          uint32_t *__restrict__ lcnt, uint32_t *__restrict__ rowbit,
                                                          CsrScal *sc) {
    __shared__ uint32_t s_w[kNW];
    uint32_t cnt3 = 0;
    unsigned long long md = 0, mr = 0;
    int bad = 0;
    for (int s = 0; s < kLineSteps; ++s) {
        const int64_t l = blockIdx.x * kLineTile + s * kTxtThreads + threadIdx.x;
        if (l >= nv) break;
        const int64_t a = off[l], z = off[l + 1], d = z - a;
        if (a < 0 || d < 0 || z > narcs || d > 0x7fffffff) {
            bad |= 1;
        } else if (d > 0) {
            cnt3 += 1u << (10 * (d <= kSmallDeg ? 0 : (d <= kLargeDeg ? 1 : 2)));
            md = max(md, (unsigned long long)d);
            atomicOr(rowbit + (a >> 5), 1u << (a & 31));
        }
        if (raw) {
            const int32_t r = raw[l];
            if (r < 0) bad |= 4;
            else mr = max(mr, (unsigned long long)r);
        }
    }
    const uint32_t c0 = block_sum(cnt3 & 1023u, s_w), c1 = block_sum((cnt3 >> 10) & 1023u, s_w),
                   c2 = block_sum(cnt3 >> 20, s_w);
    for (int o = 16; o > 0; o >>= 1) {
        md = max(md, __shfl_xor_sync(DMOLP_FULL_MASK, md, o));
        mr = max(mr, __shfl_xor_sync(DMOLP_FULL_MASK, mr, o));
    }
    bad = __reduce_or_sync(DMOLP_FULL_MASK, bad);
    if ((threadIdx.x & 31) == 0) {
        if (md) atomicMax(&sc->maxdeg, md);
        if (mr) atomicMax(&sc->maxraw, mr);
        if (bad) atomicOr(&sc->bad, bad);
    }
    if (threadIdx.x == 0) {
        lcnt[3 * blockIdx.x] = c0;
        lcnt[3 * blockIdx.x + 1] = c1;
        lcnt[3 * blockIdx.x + 2] = c2;
    }
}

// Per 4 arcs (one 16-byte load): every id in [0, nv), and every arc that does not start its row above its
// predecessor.  The rows' bits come from k_csr_rows; after bad offsets the order test is skipped (the upload
// fails anyway).  Whole warps iterate, so the predecessor of a lane's first arc comes from the lane below.
__global__ void __launch_bounds__(256) k_csr_arcs(const int32_t *__restrict__ col, int64_t narcs, int64_t nv,
                                                  const uint32_t *__restrict__ rowbit, CsrScal *sc) {
    const int lane = threadIdx.x & 31;
    const bool order = (((volatile CsrScal *)sc)->bad & 1) == 0;
    const int64_t n4 = narcs >> 2;
    const int64_t nwarp = (int64_t)gridDim.x * (blockDim.x >> 5);
    int bad = 0;
    unsigned long long viol = 0;
    // two 16-byte groups per lane and step (512 arcs per warp), their loads in flight together
    for (int64_t w0 = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 64; w0 < n4; w0 += nwarp * 64) {
        int4 q[2];
        uint32_t bits[2];
        int pre[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t i = w0 + h * 32 + lane;
            q[h] = make_int4(0, 0, 0, 0);
            bits[h] = 0xfu;
            pre[h] = 0;
            if (i < n4) {
                q[h] = __ldcs(reinterpret_cast<const int4 *>(col) + i);
                bits[h] = (__ldg(rowbit + (i >> 3)) >> ((i & 7) * 4)) & 0xfu;
                if (lane == 0 && i > 0) pre[h] = __ldg(col + 4 * i - 1);
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t i = w0 + h * 32 + lane;
            int prev = __shfl_up_sync(DMOLP_FULL_MASK, q[h].w, 1);
            if (lane == 0) prev = pre[h];
            if (i < n4) {
                const int x[4] = {q[h].x, q[h].y, q[h].z, q[h].w};
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    if ((uint32_t)x[t] >= (uint64_t)nv) bad = 2;
                    if (order && !((bits[h] >> t) & 1u) && (i > 0 || t > 0) && x[t] <= (t ? x[t - 1] : prev)) ++viol;
                }
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x < 4) {  // the last narcs % 4 arcs
        const int64_t j = 4 * n4 + threadIdx.x;
        if (j < narcs) {
            const int x = col[j];
            if ((uint32_t)x >= (uint64_t)nv) bad = 2;
            if (order && !((rowbit[j >> 5] >> (j & 31)) & 1u) && j > 0 && x <= col[j - 1]) ++viol;
        }
    }
    bad = __reduce_or_sync(DMOLP_FULL_MASK, bad);
    viol = __reduce_add_sync(DMOLP_FULL_MASK, (unsigned)viol);
    if (lane == 0) {
        if (bad) atomicOr(&sc->bad, bad);
        if (viol) atomicAdd(&sc->violations, viol);
    }
}

// Degree-class lists in ascending id order (isolated vertices in none), at the tile prefixes loff.
__global__ void __launch_bounds__(kTxtThreads) k_csr_classes(const int64_t *__restrict__ off, int64_t nv,
                                                             const int64_t *__restrict__ loff, int32_t *b0, int32_t *b1,
                                                             int32_t *b2) {
    __shared__ uint32_t s_w[kNW];
    int64_t base[3] = {loff[3 * blockIdx.x], loff[3 * blockIdx.x + 1], loff[3 * blockIdx.x + 2]};
    for (int s = 0; s < kLineSteps; ++s) {
        const int64_t l = blockIdx.x * kLineTile + s * kTxtThreads + threadIdx.x;
        if (blockIdx.x * kLineTile + s * kTxtThreads >= nv) break;  // uniform across the block
        int cls = 3;
        if (l < nv) {
            const int64_t d = off[l + 1] - off[l];
            cls = d == 0 ? 3 : (d <= kSmallDeg ? 0 : (d <= kLargeDeg ? 1 : 2));
        }
        uint32_t tot;
        const uint32_t ex = block_excl_scan(cls < 3 ? 1u << (10 * cls) : 0u, &tot, s_w);
        if (cls < 3) {
            int32_t *b = cls == 0 ? b0 : (cls == 1 ? b1 : b2);
            b[base[cls] + ((ex >> (10 * cls)) & 1023u)] = (int32_t)l;
        }
        for (int c = 0; c < 3; ++c) base[c] += (tot >> (10 * c)) & 1023u;
    }
}

// ---- host side ----

template <typename T>
bool pool_get(Pool &pool, int slot, T **p, size_t n, std::string &err) {
    *p = (T *)pool.get(slot, std::max<size_t>(n, 1) * sizeof(T), err);
    return *p != nullptr;
}

#define ING_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);               \
            return 1;                                                               \
        }                                                                           \
    } while (0)
#define ING_ALLOC(slot, ptr, n) \
    if (!pool_get(*p.pool, (slot), &(ptr), (n), err)) return 1

struct Events {  // timing of the two text passes, destroyed on every exit path
    cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};
    ~Events() {
        for (cudaEvent_t x : e)
            if (x) cudaEventDestroy(x);
    }
};

int grid_for(int64_t n, int threads) {
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, (int64_t)sms * 16));
}

}  // namespace

void *Pool::get(int slot, size_t bytes, std::string &err) {
    if (cap[slot] < bytes) {
        if (ptr[slot]) cudaFree(ptr[slot]);
        ptr[slot] = nullptr;
        cap[slot] = 0;
        const size_t want = (bytes + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
        cudaError_t e = cudaMalloc(&ptr[slot], want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ptr[slot] = nullptr;
            err = std::string("cudaMalloc (parse scratch): ") + cudaGetErrorString(e);
            return nullptr;
        }
        cap[slot] = want;
    }
    return ptr[slot];
}

size_t Pool::held() const {
    size_t t = 0;
    for (size_t c : cap) t += c;
    return t;
}

void Pool::release() {
    for (int i = 0; i < kNumSlots; ++i) {
        if (ptr[i]) cudaFree(ptr[i]);
        ptr[i] = nullptr;
        cap[i] = 0;
    }
}

void release(Parsed &p) { p = Parsed(); }

int parse(cudaStream_t st, uint8_t *d_txt, int64_t len, int64_t body0, int64_t body1, Pool &pool, Parsed &p,
          std::string &err) {
    release(p);
    p.pool = &pool;
    (void)len;
    Events ev;
    for (cudaEvent_t &e : ev.e) ING_CUDA(cudaEventCreate(&e));
    Scal *sc = nullptr;
    ING_ALLOC(kScal, sc, 1);
    p.scal = sc;
    ING_CUDA(cudaMemsetAsync(sc, 0, sizeof(Scal), st));
    const int64_t nt = body1 > body0 ? (body1 + kTileBytes - 1) / kTileBytes : 0;
    int64_t tot[2] = {0, 0};
    if (nt > 0) {
        ING_ALLOC(kTcnt, p.tcnt, (size_t)2 * nt);
        ING_ALLOC(kToff, p.toff, (size_t)2 * (nt + 1));
        ING_CUDA(cudaEventRecord(ev.e[0], st));
        k_txt_count<<<(unsigned)nt, kTxtThreads, 0, st>>>(d_txt, body0, body1, p.tcnt, sc);
        ING_CUDA(cudaEventRecord(ev.e[1], st));
        ++p.launches;
        unsigned long long nul = 0;
        ING_CUDA(cudaMemcpyAsync(&nul, &sc->nul, sizeof(nul), cudaMemcpyDeviceToHost, st));
        ING_CUDA(cudaStreamSynchronize(st));
        if (nul) {
            k_txt_nulfill<<<grid_for((body1 - body0) / 16 + 1, 256), 256, 0, st>>>(d_txt, body0, body1);
            k_txt_count<<<(unsigned)nt, kTxtThreads, 0, st>>>(d_txt, body0, body1, p.tcnt, sc);
            p.launches += 2;
        }
        k_scan<2><<<1, 1024, 0, st>>>(p.tcnt, nt, p.toff);
        ++p.launches;
        ING_CUDA(cudaMemcpyAsync(tot, p.toff + 2 * nt, sizeof(tot), cudaMemcpyDeviceToHost, st));
        ING_CUDA(cudaStreamSynchronize(st));
        ING_CUDA(cudaGetLastError());
    }
    p.nv = tot[0];
    p.ntok = tot[1];
    if (p.nv > 0x7ffffffe) {
        err = "too many vertices for int32 ids";
        return 1;
    }
    ING_ALLOC(kTok, p.tok, (size_t)p.ntok);
    ING_ALLOC(kEndTok, p.end_tok, (size_t)p.nv);
    ING_ALLOC(kBadrow, p.badrow, (size_t)p.nv);
    Scal h{};
    if (p.nv > 0) {
        ING_CUDA(cudaEventRecord(ev.e[2], st));
        k_txt_emit<<<(unsigned)nt, kTxtThreads, 0, st>>>(d_txt, body0, body1, p.nv, p.toff, p.tok, p.end_tok, sc);
        ING_CUDA(cudaEventRecord(ev.e[3], st));
        ING_CUDA(cudaMemsetAsync(p.badrow, 0, (size_t)p.nv, st));
        ++p.launches;
        if (p.ntok > 1) {
            k_tok_check<<<grid_for(p.ntok, 256), 256, 0, st>>>(p.tok, p.ntok, p.end_tok, p.nv, p.badrow, sc);
            ++p.launches;
        }
        ING_CUDA(cudaMemcpyAsync(&h, sc, sizeof(h), cudaMemcpyDeviceToHost, st));
        ING_CUDA(cudaStreamSynchronize(st));
        ING_CUDA(cudaGetLastError());
        cudaEventElapsedTime(&p.count_ms, ev.e[0], ev.e[1]);
        cudaEventElapsedTime(&p.emit_ms, ev.e[2], ev.e[3]);
    }
    if (h.bad_id) {
        err = "a neighbour id is outside [0, V)";
        return 1;
    }
    p.sorted = h.violations == 0;
    p.narcs = p.ntok;
    if (!p.sorted) {
        ING_ALLOC(kLists, p.lists, (size_t)3 * p.nv);
        k_rows_classify<<<grid_for(p.nv, 256), 256, 0, st>>>(p.end_tok, p.nv, p.badrow, p.lists, sc);
        ++p.launches;
        ING_CUDA(cudaMemcpyAsync(&h, sc, sizeof(h), cudaMemcpyDeviceToHost, st));
        ING_CUDA(cudaStreamSynchronize(st));
        p.rows_sorted = (int64_t)h.nlist[0] + h.nlist[1] + h.nlist[2];
        if (h.nlist[0]) {
            k_sort_small<<<(h.nlist[0] + 127) / 128, 128, 0, st>>>(p.tok, p.end_tok, p.lists, h.nlist[0]);
            ++p.launches;
        }
        if (h.nlist[1]) {
            k_sort_mid<<<h.nlist[1], 512, 0, st>>>(p.tok, p.end_tok, p.lists + p.nv);
            ++p.launches;
        }
        if (h.nlist[2]) {
            ING_ALLOC(kTmp, p.tmp, (size_t)p.ntok);
            k_sort_big<<<h.nlist[2], 1024, 0, st>>>(p.tok, p.tmp, p.end_tok, p.lists + 2 * p.nv);
            ++p.launches;
        }
        const int64_t ntt = (p.ntok + kTokTile - 1) / kTokTile;
        ING_ALLOC(kTcnt, p.tcnt, (size_t)ntt);  // the text tiles' counters are no longer needed
        ING_ALLOC(kToff, p.toff, (size_t)ntt + 1);
        ING_ALLOC(kKeptpos, p.keptpos, (size_t)p.ntok + 1);
        k_keep_count<<<(unsigned)ntt, kTxtThreads, 0, st>>>(p.tok, p.ntok, p.tcnt);
        k_scan<1><<<1, 1024, 0, st>>>(p.tcnt, ntt, p.toff);
        k_keep_pos<<<(unsigned)ntt, kTxtThreads, 0, st>>>(p.tok, p.ntok, p.toff, p.keptpos);
        p.launches += 3;
        ING_CUDA(cudaMemcpyAsync(&p.narcs, p.keptpos + p.ntok, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    }
    const int64_t nlt = (p.nv + kLineTile - 1) / kLineTile;
    uint32_t *lcnt = nullptr;
    ING_ALLOC(kLcnt, lcnt, (size_t)3 * nlt);
    ING_ALLOC(kLoff, p.loff, (size_t)3 * (nlt + 1));
    int64_t nb[3] = {0, 0, 0};
    if (nlt > 0) {
        k_lines_count<<<(unsigned)nlt, kTxtThreads, 0, st>>>(p.end_tok, p.keptpos, p.nv, lcnt, sc);
        k_scan<3><<<1, 1024, 0, st>>>(lcnt, nlt, p.loff);
        p.launches += 2;
        ING_CUDA(cudaMemcpyAsync(nb, p.loff + 3 * nlt, sizeof(nb), cudaMemcpyDeviceToHost, st));
        ING_CUDA(cudaMemcpyAsync(&h, sc, sizeof(h), cudaMemcpyDeviceToHost, st));
    }
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        err = std::string("ingest: ") + cudaGetErrorString(e);
        return 1;
    }
    ING_CUDA(cudaGetLastError());
    for (int c = 0; c < 3; ++c) p.nb[c] = nb[c];
    p.maxdeg = (int64_t)h.maxdeg;
    p.maxraw = (int64_t)h.maxraw;
    if (p.maxraw > 0x7fffffff) {
        err = "a line has more than 2^31-1 tokens";
        return 1;
    }
    return 0;
}

int check_csr(cudaStream_t st, const int64_t *off, const int32_t *col, const int32_t *raw, int64_t nv, int64_t narcs,
              Pool &pool, CsrInfo &out, std::string &err) {
    out = CsrInfo();
    CsrScal *sc = nullptr;
    if (!pool_get(pool, kScal, &sc, 1, err)) return 1;
    ING_CUDA(cudaMemsetAsync(sc, 0, sizeof(CsrScal), st));
    const int64_t nlt = (nv + kLineTile - 1) / kLineTile;
    const int64_t nwords = (narcs + 31) / 32;
    uint32_t *lcnt = nullptr, *rowbit = nullptr;
    int64_t *loff = nullptr;
    if (!pool_get(pool, kLcnt, &lcnt, (size_t)3 * nlt, err) || !pool_get(pool, kLoff, &loff, (size_t)3 * (nlt + 1), err) ||
        !pool_get(pool, kKeptpos, &rowbit, (size_t)nwords, err))
        return 1;
    if (nwords) ING_CUDA(cudaMemsetAsync(rowbit, 0, (size_t)nwords * sizeof(uint32_t), st));
    int64_t nb[3] = {0, 0, 0};
    if (nlt > 0) {
        k_csr_rows<<<(unsigned)nlt, kTxtThreads, 0, st>>>(off, raw, nv, narcs, lcnt, rowbit, sc);
        k_scan<3><<<1, 1024, 0, st>>>(lcnt, nlt, loff);
        out.launches += 2;
    }
    if (narcs > 0) {
        k_csr_arcs<<<grid_for(narcs / 8 + 1, 256), 256, 0, st>>>(col, narcs, nv, rowbit, sc);
        ++out.launches;
    }
    CsrScal h{};
    ING_CUDA(cudaMemcpyAsync(&h, sc, sizeof(h), cudaMemcpyDeviceToHost, st));
    if (nlt > 0) ING_CUDA(cudaMemcpyAsync(nb, loff + 3 * nlt, sizeof(nb), cudaMemcpyDeviceToHost, st));
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        err = std::string("upload check: ") + cudaGetErrorString(e);
        return 1;
    }
    ING_CUDA(cudaGetLastError());
    out.bad = h.bad;
    out.sorted = h.violations == 0;
    out.maxdeg = (int64_t)h.maxdeg;
    out.maxraw = (int64_t)h.maxraw;
    for (int c = 0; c < 3; ++c) out.nb[c] = nb[c];
    out.loff = loff;
    return 0;
}

int csr_classes(cudaStream_t st, const int64_t *off, int64_t nv, const CsrInfo &info, int32_t *const bucket[3],
                std::string &err) {
    const int64_t nlt = (nv + kLineTile - 1) / kLineTile;
    if (nlt > 0)
        k_csr_classes<<<(unsigned)nlt, kTxtThreads, 0, st>>>(off, nv, info.loff, bucket[0], bucket[1], bucket[2]);
    ING_CUDA(cudaGetLastError());
    return 0;
}

int build(cudaStream_t st, Parsed &p, int64_t *off, int32_t *col, int32_t *raw, int32_t *const bucket[3],
          std::string &err) {
    const int64_t nlt = (p.nv + kLineTile - 1) / kLineTile;
    if (nlt > 0) {
        k_lines_emit<<<(unsigned)nlt, kTxtThreads, 0, st>>>(p.end_tok, p.keptpos, p.nv, p.loff, off, raw, bucket[0],
                                                            bucket[1], bucket[2]);
        ++p.launches;
    } else {
        ING_CUDA(cudaMemsetAsync(off, 0, sizeof(int64_t), st));
    }
    if (p.ntok > 0) {
        if (p.sorted) k_col_copy<<<grid_for(p.ntok / 4 + 1, 256), 256, 0, st>>>(p.tok, p.ntok, col);
        else k_keep_compact<<<grid_for(p.ntok, 256), 256, 0, st>>>(p.tok, p.ntok, p.keptpos, col);
        ++p.launches;
    }
    ING_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace ingest
}  // namespace dmolp
