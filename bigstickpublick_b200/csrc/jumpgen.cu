// On-device generation of the jump tables (the set-up stage that BIGSTICK
// runs on the host: weld/master1bodyjumps/master2bodyjumps,
// src/bjumplib_weld.f90:296-809, src/bjumplib_master.f90:436-1196, and the
// jump sort sort1bjumps, src/bsortjumpslib.f90:21-290).
//
// A species is given by its Slater determinants (occupation bitmasks), their
// pstart/nstart values and its sectors.  The jumps of a sector jump are the
// reference's, in the same order as the host table builder writes them:
// source SD ascending, then the annihilated state k, then the created state i
// (one-body), or the annihilated pair (k<l) and the created pair (i<j) of the
// same (M, parity) section (two-body; inside a sector only isd >= fsd).
//   * count: one thread per (sector jump, source SD) counts its jumps;
//   * an exclusive scan of the counts gives every thread its output slot in
//     sector-jump-major order, so the layout needs no sort;
//   * write: the same threads enumerate again and write isd, fsd, labels and
//     phases.
// The PN bundles' ranges are then sorted by the reference's shell sort with
// its fixed stride table; within one stride pass the interleaved
// subsequences are independent, so the threads of a CTA take them in
// parallel and the result is the sequential algorithm's, element for element.

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "bsg_internal.h"
#include "ref_order.h"

struct bsg_jumpgen {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    int32_t nsps = 0, nl = 0;
    int64_t nsd = 0;
    int32_t nsectors = 0;
    std::vector<int64_t> sec_start, sec_end;     // 1-based SD ranges
    // device
    bsg::DevBuf bits, xstart, sd_sector, dense, pair_at, pair_sec, sec_first, sec_me, cre_off, cre_list;
    double last_ms = 0.0;
};

namespace bsg {

constexpr int kMaxJumpSps = 22;   // dense SD lookup of 2^nsps entries

__device__ __forceinline__ int jg_nbelow(uint64_t bits, int q) {
    return __popcll(q == 0 ? 0ull : (bits & ((1ull << q) - 1ull)));
}
__device__ __forceinline__ int jg_label(int nl, int q) { return q < nl ? -(q + 1) : (q - nl + 1); }
// a+_i a_k |s>: sign relative to the ascending-label product
__device__ __forceinline__ int jg_phase1(uint64_t bits, int i, int k) {
    if (i == k) return 1;
    const int p = jg_nbelow(bits, k) + jg_nbelow(bits & ~(1ull << k), i);
    return (p & 1) ? -1 : 1;
}
// a+_i a+_j a_l a_k |s>, i<j, k<l
__device__ __forceinline__ int jg_phase2(uint64_t bits, int i, int j, int k, int l) {
    int p = jg_nbelow(bits, k);
    uint64_t b = bits & ~(1ull << k);
    p += jg_nbelow(b, l);
    b &= ~(1ull << l);
    p += jg_nbelow(b, j);
    b |= (1ull << j);
    p += jg_nbelow(b, i);
    return (p & 1) ? -1 : 1;
}

struct JG {
    int32_t nsps, nl;
    const uint64_t *bits;
    const int64_t *xstart;
    const int32_t *sd_sector;
    const int32_t *dense;          // bits -> SD index (0-based) or -1
    // two-body pair tables (pairs q1 < q2 in the reference's section order)
    const int32_t *pair_at;        // [q1*nsps + q2] -> pair index (1-based)
    const int32_t *pair_sec;       // [pair-1] -> section
    const int64_t *sec_first;      // first pair index (1-based) of each section
    const int64_t *sec_me;         // first label - 1 of each section (triangle packing)
    const int32_t *cre_off;        // creation pairs of each section: cre_list[cre_off[s] .. cre_off[s+1])
    const int2 *cre_list;          // (i, j), i < j, in (i, j) order
};

// items: (sector jump or sector j, source SD); item t of j is SD sd0[j] + (t - item_off[j])
__device__ __forceinline__ int jg_find(const int64_t *__restrict__ item_off, int n, int64_t t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (item_off[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <bool WRITE>
__global__ void k_jumps1(const JG g, const int32_t *__restrict__ fs, const int64_t *__restrict__ sd0,
                         const int64_t *__restrict__ item_off, int nsj, int64_t nitems, int64_t *__restrict__ cnt,
                         const int64_t *__restrict__ out_off, int64_t *__restrict__ isd, int64_t *__restrict__ fsd,
                         int16_t *__restrict__ cop, int16_t *__restrict__ dop, int8_t *__restrict__ phase) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nitems; t += (int64_t)gridDim.x * blockDim.x) {
        const int j = jg_find(item_off, nsj, t);
        const int64_t sd = sd0[j] + (t - item_off[j]);
        const int target = fs[j];
        const uint64_t bits = g.bits[sd];
        int64_t o = WRITE ? out_off[t] : 0;
        int64_t n = 0;
        for (int k = 0; k < g.nsps; ++k) {
            if (!(bits >> k & 1ull)) continue;
            for (int i = 0; i < g.nsps; ++i) {
                if (i != k && (bits >> i & 1ull)) continue;
                const uint64_t nb = (bits & ~(1ull << k)) | (1ull << i);
                const int f = g.dense[nb];
                if (f < 0 || g.sd_sector[f] != target) continue;
                if (WRITE) {
                    isd[o] = g.xstart[sd];
                    fsd[o] = g.xstart[f];
                    cop[o] = (int16_t)jg_label(g.nl, i);
                    dop[o] = (int16_t)jg_label(g.nl, k);
                    phase[o] = (int8_t)jg_phase1(bits, i, k);
                    ++o;
                }
                ++n;
            }
        }
        if (!WRITE) cnt[t] = n;
    }
}

template <bool WRITE>
__global__ void k_jumps2(const JG g, const int32_t *__restrict__ sec, const int64_t *__restrict__ sd0,
                         const int64_t *__restrict__ item_off, int nsec, int64_t nitems, int64_t *__restrict__ cnt,
                         const int64_t *__restrict__ out_off, int64_t *__restrict__ isd, int64_t *__restrict__ fsd,
                         int32_t *__restrict__ op, int8_t *__restrict__ phase) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nitems; t += (int64_t)gridDim.x * blockDim.x) {
        const int j = jg_find(item_off, nsec, t);
        const int64_t sd = sd0[j] + (t - item_off[j]);
        const int target = sec[j];
        const uint64_t bits = g.bits[sd];
        int64_t o = WRITE ? out_off[t] : 0;
        int64_t n = 0;
        for (int k = 0; k < g.nsps; ++k) {
            if (!(bits >> k & 1ull)) continue;
            for (int l = k + 1; l < g.nsps; ++l) {
                if (!(bits >> l & 1ull)) continue;
                const uint64_t rest = bits & ~(1ull << k) & ~(1ull << l);
                const int dpair = g.pair_at[k * g.nsps + l];
                const int s = g.pair_sec[dpair - 1];
                for (int c = g.cre_off[s]; c < g.cre_off[s + 1]; ++c) {
                    const int2 ij = g.cre_list[c];
                    if ((rest >> ij.x & 1ull) || (rest >> ij.y & 1ull)) continue;
                    const uint64_t nb = rest | (1ull << ij.x) | (1ull << ij.y);
                    const int f = g.dense[nb];
                    if (f < 0 || g.sd_sector[f] != target) continue;
                    if (sd < f) continue;  // inside a sector: keep isd >= fsd
                    if (WRITE) {
                        const int cpair = g.pair_at[ij.x * g.nsps + ij.y];
                        const int64_t iref = g.sec_first[s] - 1, istart = g.sec_me[s];
                        const int64_t hi = max(cpair, dpair), lo = min(cpair, dpair);
                        isd[o] = g.xstart[sd];
                        fsd[o] = g.xstart[f];
                        op[o] = (int32_t)(istart + (hi - iref) * (hi - iref - 1) / 2 + lo - iref);
                        phase[o] = (int8_t)jg_phase2(bits, ij.x, ij.y, k, l);
                        ++o;
                    }
                    ++n;
                }
            }
        }
        if (!WRITE) cnt[t] = n;
    }
}

// exclusive scan of n int64 counts (tiles of 1024, tile sums scanned by the
// same routine)
constexpr int kScanTile = 1024;
__global__ void k_scan_tiles(const int64_t *__restrict__ in, int64_t *__restrict__ out, int64_t n,
                             int64_t *__restrict__ tile_sum) {
    __shared__ int64_t s[kScanTile];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    for (int e = threadIdx.x; e < kScanTile; e += blockDim.x) s[e] = (base + e < n) ? in[base + e] : 0;
    __syncthreads();
    // Hillis-Steele over the tile (inclusive), then shift
    for (int d = 1; d < kScanTile; d <<= 1) {
        int64_t v[kScanTile / 256];
        for (int r = 0; r < kScanTile / 256; ++r) {
            const int e = threadIdx.x + 256 * r;
            v[r] = (e >= d) ? s[e - d] : 0;
        }
        __syncthreads();
        for (int r = 0; r < kScanTile / 256; ++r) s[threadIdx.x + 256 * r] += v[r];
        __syncthreads();
    }
    for (int e = threadIdx.x; e < kScanTile; e += blockDim.x)
        if (base + e < n) out[base + e] = (e == 0 ? 0 : s[e - 1]);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = s[kScanTile - 1];
}
__global__ void k_scan_add(int64_t *__restrict__ out, int64_t n, const int64_t *__restrict__ tile_off) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        out[e] += tile_off[e / kScanTile];
}

static cudaError_t scan_i64(const int64_t *in, int64_t *out, int64_t n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    int64_t *sum = nullptr, *off = nullptr;
    cudaError_t e = cudaMallocAsync(&sum, sizeof(int64_t) * tiles, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&off, sizeof(int64_t) * tiles, s);
    if (e == cudaSuccess) {
        k_scan_tiles<<<(unsigned)tiles, 256, 0, s>>>(in, out, n, sum);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && tiles > 1) {
        e = scan_i64(sum, off, tiles, s);
        if (e == cudaSuccess) {
            k_scan_add<<<(unsigned)std::min<int64_t>((n + 255) / 256, 65535), 256, 0, s>>>(out, n, off);
            e = cudaGetLastError();
        }
    }
    if (sum) cudaFreeAsync(sum, s);
    if (off) cudaFreeAsync(off, s);
    return e;
}

// sort1bjumps: shell sort of each range by key, the rest carried along, with
// the reference's stride table; one CTA per range, the subsequences of a
// stride pass in parallel
__constant__ int64_t c_strides[28] = {23422578909LL, 10410035071LL, 4626682254LL, 2056303224LL, 913912544LL,
                                      406183353LL,   180525935LL,   80233749LL,   35659463LL,   15848650LL,
                                      7043844LL,     3130597LL,     1391376LL,    463792LL,     198768LL,
                                      86961LL,       33936LL,       13776LL,      4592LL,       1968LL,
                                      861LL,         336LL,         112LL,        48LL,         21LL,
                                      7LL,           3LL,           1LL};
__global__ void k_shell_sort(const int64_t *__restrict__ start, const int64_t *__restrict__ len, int64_t *key,
                             int64_t *other, int16_t *cop, int16_t *dop, int8_t *ph) {
    const int64_t s0 = start[blockIdx.x], ndim = len[blockIdx.x];
    int64_t *K = key + s0, *O = other + s0;
    int16_t *C = cop + s0, *D = dop + s0;
    int8_t *P = ph + s0;
    for (int ks = 0; ks < 28; ++ks) {
        const int64_t stride = c_strides[ks];
        if (stride > ndim) continue;
        for (int64_t off = threadIdx.x; off < stride; off += blockDim.x) {
            // 1-based: j = off+stride+1, ..., ndim step stride
            for (int64_t j = off + stride + 1; j <= ndim; j += stride) {
                const int64_t s_o = O[j - 1], s_k = K[j - 1];
                const int16_t s_c = C[j - 1], s_d = D[j - 1];
                const int8_t s_p = P[j - 1];
                int64_t k = j, i = k - stride;
                while (i > 0) {
                    if (K[i - 1] <= s_k) break;
                    O[k - 1] = O[i - 1]; K[k - 1] = K[i - 1];
                    C[k - 1] = C[i - 1]; D[k - 1] = D[i - 1]; P[k - 1] = P[i - 1];
                    k = i;
                    i -= stride;
                }
                O[k - 1] = s_o; K[k - 1] = s_k; C[k - 1] = s_c; D[k - 1] = s_d; P[k - 1] = s_p;
            }
        }
        __syncthreads();
    }
}

}  // namespace bsg

using namespace bsg;

namespace {

int jerr(bsg_jumpgen *g, int code, const std::string &m) {
    g->last_error = m;
    return code;
}

JG jg_view(const bsg_jumpgen *g) {
    JG v;
    v.nsps = g->nsps;
    v.nl = g->nl;
    v.bits = (const uint64_t *)g->bits.p;
    v.xstart = (const int64_t *)g->xstart.p;
    v.sd_sector = (const int32_t *)g->sd_sector.p;
    v.dense = (const int32_t *)g->dense.p;
    v.pair_at = (const int32_t *)g->pair_at.p;
    v.pair_sec = (const int32_t *)g->pair_sec.p;
    v.sec_first = (const int64_t *)g->sec_first.p;
    v.sec_me = (const int64_t *)g->sec_me.p;
    v.cre_off = (const int32_t *)g->cre_off.p;
    v.cre_list = (const int2 *)g->cre_list.p;
    return v;
}

// scratch device buffer (freed at scope exit)
struct Scratch {
    void *p = nullptr;
    ~Scratch() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 16); }
};

cudaError_t up(Scratch &d, const void *h, size_t bytes, cudaStream_t s) {
    cudaError_t e = d.alloc(bytes);
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(d.p, h, bytes, cudaMemcpyHostToDevice, s);
    return e;
}

// the shared driver of the one- and two-body generators: items of group j
// are the SDs of sector src[j]; count, scan, then (outputs given) write
template <typename CountFn, typename WriteFn>
int run_groups(bsg_jumpgen *g, int ngroups, const int32_t *src, int64_t *starts, bool write, CountFn count,
               WriteFn writefn, Scratch &out_off, int64_t &total) {
    std::vector<int64_t> sd0(ngroups), item_off(ngroups + 1, 0);
    for (int j = 0; j < ngroups; ++j) {
        if (src[j] < 0 || src[j] >= g->nsectors) return jerr(g, BSG_ERR_ARG, "sector index out of range");
        sd0[j] = g->sec_start[src[j]] - 1;
        item_off[j + 1] = item_off[j] + (g->sec_end[src[j]] - g->sec_start[src[j]] + 1);
    }
    const int64_t nitems = item_off[ngroups];
    cudaStream_t s = g->stream;
    Scratch d_sd0, d_off, d_cnt;
    cudaError_t e = up(d_sd0, sd0.data(), 8 * sd0.size(), s);
    if (e == cudaSuccess) e = up(d_off, item_off.data(), 8 * item_off.size(), s);
    if (e == cudaSuccess) e = d_cnt.alloc(8 * (size_t)std::max<int64_t>(nitems, 1));
    if (e == cudaSuccess) e = out_off.alloc(8 * (size_t)(nitems + 1));
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((nitems + 255) / 256, 65535));
    if (e == cudaSuccess && nitems) e = count(grid, (const int64_t *)d_sd0.p, (const int64_t *)d_off.p, nitems,
                                              (int64_t *)d_cnt.p);
    if (e == cudaSuccess) e = scan_i64((const int64_t *)d_cnt.p, (int64_t *)out_off.p, nitems, s);
    // group starts and the total
    std::vector<int64_t> last(2, 0);
    if (e == cudaSuccess && nitems) {
        e = cudaMemcpyAsync(&last[0], (int64_t *)out_off.p + nitems - 1, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&last[1], (int64_t *)d_cnt.p + nitems - 1, 8, cudaMemcpyDeviceToHost, s);
    }
    std::vector<int64_t> gs(ngroups + 1, 0);
    for (int j = 0; j < ngroups && e == cudaSuccess; ++j)
        if (item_off[j] < nitems)
            e = cudaMemcpyAsync(&gs[j], (int64_t *)out_off.p + item_off[j], 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return jerr(g, BSG_ERR_CUDA, std::string("jump count: ") + cudaGetErrorString(e));
    total = nitems ? last[0] + last[1] : 0;
    for (int j = 0; j < ngroups; ++j)
        if (item_off[j] >= nitems) gs[j] = total;
    gs[ngroups] = total;
    if (starts) std::copy(gs.begin(), gs.end(), starts);
    if (write && total > 0) {
        e = writefn(grid, (const int64_t *)d_sd0.p, (const int64_t *)d_off.p, nitems, (const int64_t *)out_off.p);
        if (e != cudaSuccess) return jerr(g, BSG_ERR_CUDA, std::string("jump write: ") + cudaGetErrorString(e));
    }
    return BSG_OK;
}

}  // namespace

extern "C" {

int bsg_jumpgen_create(int device, const bsg_species *sp, bsg_jumpgen **out) {
    if (!out || !sp) return BSG_ERR_ARG;
    *out = nullptr;
    if (sp->nsps < 1 || sp->nsps > kMaxJumpSps || sp->nl < 0 || sp->nl > sp->nsps || sp->nsd < 0 || !sp->m2 ||
        !sp->par || (sp->nsd > 0 && (!sp->sd_bits || !sp->xstart)) || sp->nsectors < 0 ||
        (sp->nsectors > 0 && (!sp->sector_start || !sp->sector_end)))
        return BSG_ERR_ARG;
    bsg_jumpgen *g = new bsg_jumpgen();
    g->device = device;
    g->nsps = sp->nsps;
    g->nl = sp->nl;
    g->nsd = sp->nsd;
    g->nsectors = sp->nsectors;
    g->sec_start.assign(sp->sector_start, sp->sector_start + sp->nsectors);
    g->sec_end.assign(sp->sector_end, sp->sector_end + sp->nsectors);
    const int ns = sp->nsps;
    // SD -> sector and the dense lookup, validated
    std::vector<int32_t> sd_sector(sp->nsd, -1), dense((size_t)1 << ns, -1);
    for (int s = 0; s < sp->nsectors; ++s) {
        if (g->sec_start[s] < 1 || g->sec_end[s] > sp->nsd || g->sec_end[s] < g->sec_start[s] - 1) {
            delete g;
            return BSG_ERR_ARG;
        }
        for (int64_t k = g->sec_start[s] - 1; k < g->sec_end[s]; ++k) sd_sector[k] = s;
    }
    for (int64_t k = 0; k < sp->nsd; ++k) {
        const uint64_t b = sp->sd_bits[k];
        if (sd_sector[k] < 0 || (b >> ns) != 0 || dense[b] >= 0) {
            delete g;
            return BSG_ERR_ARG;
        }
        dense[b] = (int32_t)k;
    }
    // pairs q1 < q2 in the reference's order: generated with the higher state
    // outer (count_create_pairs, src/btbme.f90:208-308), then sortpair
    // (:548-703) into sections of equal M = (m1+m2)/2 and parity, M
    // descending, parity 1 then 2
    struct P { int q1, q2, M, pidx; };
    std::vector<P> v;
    for (int q2 = 1; q2 < ns; ++q2)
        for (int q1 = 0; q1 < q2; ++q1) {
            const int pp = sp->par[q1] * sp->par[q2];
            v.push_back(P{q1, q2, (sp->m2[q1] + sp->m2[q2]) / 2, pp > 0 ? 1 : 2});
        }
    bsg_order::sortpair(v);
    std::vector<int32_t> pair_at((size_t)ns * ns, 0), pair_sec(v.size());
    std::vector<int64_t> sec_first, sec_me;
    int64_t nme = 0, secn = 0;
    for (size_t i = 0; i < v.size(); ++i) {
        if (i == 0 || v[i].M != v[i - 1].M || v[i].pidx != v[i - 1].pidx) {
            if (!sec_first.empty()) nme += secn * (secn + 1) / 2;
            sec_first.push_back((int64_t)i + 1);
            sec_me.push_back(nme);
            secn = 0;
        }
        ++secn;
        pair_at[(size_t)v[i].q1 * ns + v[i].q2] = (int32_t)i + 1;
        pair_sec[i] = (int32_t)sec_first.size() - 1;
    }
    // creation pairs of each section in (i, j) order
    std::vector<std::vector<int2>> by(sec_first.size());
    for (int i = 0; i < ns; ++i)
        for (int j = i + 1; j < ns; ++j) by[pair_sec[pair_at[(size_t)i * ns + j] - 1]].push_back(make_int2(i, j));
    std::vector<int32_t> cre_off(1, 0);
    std::vector<int2> cre_list;
    for (auto &b : by) {
        cre_list.insert(cre_list.end(), b.begin(), b.end());
        cre_off.push_back((int32_t)cre_list.size());
    }
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    auto upb = [&](DevBuf &b, const void *h, size_t bytes) {
        if (e != cudaSuccess) return;
        e = cudaMalloc(&b.p, bytes ? bytes : 16);
        b.bytes = bytes;
        if (e == cudaSuccess && bytes) e = cudaMemcpy(b.p, h, bytes, cudaMemcpyHostToDevice);
    };
    upb(g->bits, sp->sd_bits, 8 * (size_t)sp->nsd);
    upb(g->xstart, sp->xstart, 8 * (size_t)sp->nsd);
    upb(g->sd_sector, sd_sector.data(), 4 * sd_sector.size());
    upb(g->dense, dense.data(), 4 * dense.size());
    upb(g->pair_at, pair_at.data(), 4 * pair_at.size());
    upb(g->pair_sec, pair_sec.data(), 4 * pair_sec.size());
    upb(g->sec_first, sec_first.data(), 8 * sec_first.size());
    upb(g->sec_me, sec_me.data(), 8 * sec_me.size());
    upb(g->cre_off, cre_off.data(), 4 * cre_off.size());
    upb(g->cre_list, cre_list.data(), sizeof(int2) * cre_list.size());
    if (e != cudaSuccess) {
        bsg_jumpgen_destroy(g);
        return e == cudaErrorMemoryAllocation ? BSG_ERR_NOMEM : BSG_ERR_CUDA;
    }
    *out = g;
    return BSG_OK;
}

int bsg_jumpgen_destroy(bsg_jumpgen *g) {
    if (!g) return BSG_OK;
    cudaSetDevice(g->device);
    DevBuf *b[] = {&g->bits, &g->xstart, &g->sd_sector, &g->dense, &g->pair_at, &g->pair_sec, &g->sec_first,
                   &g->sec_me, &g->cre_off, &g->cre_list};
    for (DevBuf *x : b)
        if (x->p) cudaFree(x->p);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
    return BSG_OK;
}

int bsg_jumpgen_last_error(const bsg_jumpgen *g, char *buf, size_t len) {
    if (!g || !buf || !len) return BSG_ERR_ARG;
    std::snprintf(buf, len, "%s", g->last_error.c_str());
    return BSG_OK;
}

int bsg_jumpgen_one(bsg_jumpgen *g, int nsj, const int32_t *is, const int32_t *fs, int64_t *starts, int64_t *isd,
                    int64_t *fsd, int16_t *cop, int16_t *dop, int8_t *phase, double *kernel_ms) {
    if (!g) return BSG_ERR_ARG;
    if (nsj < 0 || (nsj > 0 && (!is || !fs)) || !starts) return jerr(g, BSG_ERR_ARG, "bsg_jumpgen_one: bad arguments");
    const bool write = isd && fsd && cop && dop && phase;
    cudaSetDevice(g->device);
    for (int j = 0; j < nsj; ++j)
        if (fs[j] < 0 || fs[j] >= g->nsectors) return jerr(g, BSG_ERR_ARG, "final sector out of range");
    cudaStream_t s = g->stream;
    Scratch d_fs, oi, of, oc, od, op;
    cudaError_t e = up(d_fs, fs, 4 * (size_t)nsj, s);
    if (e != cudaSuccess) return jerr(g, BSG_ERR_CUDA, "upload");
    const JG v = jg_view(g);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    int64_t total = 0;
    Scratch out_off;
    auto count = [&](unsigned grid, const int64_t *sd0, const int64_t *ioff, int64_t nitems, int64_t *cnt) {
        k_jumps1<false><<<grid, 256, 0, s>>>(v, (const int32_t *)d_fs.p, sd0, ioff, nsj, nitems, cnt, nullptr,
                                             nullptr, nullptr, nullptr, nullptr, nullptr);
        return cudaGetLastError();
    };
    auto writefn = [&](unsigned grid, const int64_t *sd0, const int64_t *ioff, int64_t nitems, const int64_t *ooff) {
        cudaError_t r = oi.alloc(8 * (size_t)total);
        if (r == cudaSuccess) r = of.alloc(8 * (size_t)total);
        if (r == cudaSuccess) r = oc.alloc(2 * (size_t)total);
        if (r == cudaSuccess) r = od.alloc(2 * (size_t)total);
        if (r == cudaSuccess) r = op.alloc((size_t)total);
        if (r != cudaSuccess) return r;
        k_jumps1<true><<<grid, 256, 0, s>>>(v, (const int32_t *)d_fs.p, sd0, ioff, nsj, nitems, nullptr, ooff,
                                            (int64_t *)oi.p, (int64_t *)of.p, (int16_t *)oc.p, (int16_t *)od.p,
                                            (int8_t *)op.p);
        return cudaGetLastError();
    };
    int st = run_groups(g, nsj, is, starts, write, count, writefn, out_off, total);
    if (st) return st;
    cudaEventRecord(e1, s);
    if (write && total > 0) {
        e = cudaMemcpyAsync(isd, oi.p, 8 * (size_t)total, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(fsd, of.p, 8 * (size_t)total, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(cop, oc.p, 2 * (size_t)total, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dop, od.p, 2 * (size_t)total, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(phase, op.p, (size_t)total, cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (kernel_ms) *kernel_ms = ms;
    if (e != cudaSuccess) return jerr(g, BSG_ERR_CUDA, std::string("bsg_jumpgen_one: ") + cudaGetErrorString(e));
    return BSG_OK;
}

int bsg_jumpgen_two(bsg_jumpgen *g, int nsec, const int32_t *sec, int64_t *starts, int64_t *isd, int64_t *fsd,
                    int32_t *opl, int8_t *phase, double *kernel_ms) {
    if (!g) return BSG_ERR_ARG;
    if (nsec < 0 || (nsec > 0 && !sec) || !starts) return jerr(g, BSG_ERR_ARG, "bsg_jumpgen_two: bad arguments");
    const bool write = isd && fsd && opl && phase;
    cudaSetDevice(g->device);
    cudaStream_t s = g->stream;
    Scratch d_sec, oi, of, oo, op;
    cudaError_t e = up(d_sec, sec, 4 * (size_t)nsec, s);
    if (e != cudaSuccess) return jerr(g, BSG_ERR_CUDA, "upload");
    const JG v = jg_view(g);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    int64_t total = 0;
    Scratch out_off;
    auto count = [&](unsigned grid, const int64_t *sd0, const int64_t *ioff, int64_t nitems, int64_t *cnt) {
        k_jumps2<false><<<grid, 256, 0, s>>>(v, (const int32_t *)d_sec.p, sd0, ioff, nsec, nitems, cnt, nullptr,
                                             nullptr, nullptr, nullptr, nullptr);
        return cudaGetLastError();
    };
    auto writefn = [&](unsigned grid, const int64_t *sd0, const int64_t *ioff, int64_t nitems, const int64_t *ooff) {
        cudaError_t r = oi.alloc(8 * (size_t)total);
        if (r == cudaSuccess) r = of.alloc(8 * (size_t)total);
        if (r == cudaSuccess) r = oo.alloc(4 * (size_t)total);
        if (r == cudaSuccess) r = op.alloc((size_t)total);
        if (r != cudaSuccess) return r;
        k_jumps2<true><<<grid, 256, 0, s>>>(v, (const int32_t *)d_sec.p, sd0, ioff, nsec, nitems, nullptr, ooff,
                                            (int64_t *)oi.p, (int64_t *)of.p, (int32_t *)oo.p, (int8_t *)op.p);
        return cudaGetLastError();
    };
    int st = run_groups(g, nsec, sec, starts, write, count, writefn, out_off, total);
    if (st) return st;
    cudaEventRecord(e1, s);
    if (write && total > 0) {
        e = cudaMemcpyAsync(isd, oi.p, 8 * (size_t)total, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(fsd, of.p, 8 * (size_t)total, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(opl, oo.p, 4 * (size_t)total, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(phase, op.p, (size_t)total, cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (kernel_ms) *kernel_ms = ms;
    if (e != cudaSuccess) return jerr(g, BSG_ERR_CUDA, std::string("bsg_jumpgen_two: ") + cudaGetErrorString(e));
    return BSG_OK;
}

int bsg_jumpgen_sort1(bsg_jumpgen *g, int nr, const int64_t *start, const int64_t *len, int by_fsd, int64_t n,
                      int64_t *isd, int64_t *fsd, int16_t *cop, int16_t *dop, int8_t *phase, double *kernel_ms) {
    if (!g) return BSG_ERR_ARG;
    if (nr < 0 || n < 0 || (nr > 0 && (!start || !len)) || (n > 0 && (!isd || !fsd || !cop || !dop || !phase)))
        return jerr(g, BSG_ERR_ARG, "bsg_jumpgen_sort1: bad arguments");
    // ranges inside the arrays and pairwise disjoint (a CTA per range)
    std::vector<std::pair<int64_t, int64_t>> r;
    for (int i = 0; i < nr; ++i) {
        if (start[i] < 0 || len[i] < 0 || start[i] + len[i] > n)
            return jerr(g, BSG_ERR_ARG, "bsg_jumpgen_sort1: range outside the arrays");
        if (len[i] > 1) r.push_back({start[i], len[i]});
    }
    std::sort(r.begin(), r.end());
    for (size_t i = 1; i < r.size(); ++i)
        if (r[i].first < r[i - 1].first + r[i - 1].second)
            return jerr(g, BSG_ERR_ARG, "bsg_jumpgen_sort1: ranges overlap");
    cudaSetDevice(g->device);
    cudaStream_t s = g->stream;
    std::vector<int64_t> st0(r.size()), ln(r.size());
    for (size_t i = 0; i < r.size(); ++i) { st0[i] = r[i].first; ln[i] = r[i].second; }
    Scratch d_st, d_ln, di, df, dc, dd, dp;
    cudaError_t e = up(d_st, st0.data(), 8 * st0.size(), s);
    if (e == cudaSuccess) e = up(d_ln, ln.data(), 8 * ln.size(), s);
    if (e == cudaSuccess) e = up(di, isd, 8 * (size_t)n, s);
    if (e == cudaSuccess) e = up(df, fsd, 8 * (size_t)n, s);
    if (e == cudaSuccess) e = up(dc, cop, 2 * (size_t)n, s);
    if (e == cudaSuccess) e = up(dd, dop, 2 * (size_t)n, s);
    if (e == cudaSuccess) e = up(dp, phase, (size_t)n, s);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    if (e == cudaSuccess && !r.empty()) {
        int64_t *key = by_fsd ? (int64_t *)df.p : (int64_t *)di.p;
        int64_t *oth = by_fsd ? (int64_t *)di.p : (int64_t *)df.p;
        k_shell_sort<<<(unsigned)r.size(), 256, 0, s>>>((const int64_t *)d_st.p, (const int64_t *)d_ln.p, key, oth,
                                                         (int16_t *)dc.p, (int16_t *)dd.p, (int8_t *)dp.p);
        e = cudaGetLastError();
    }
    cudaEventRecord(e1, s);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(isd, di.p, 8 * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(fsd, df.p, 8 * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(cop, dc.p, 2 * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(dop, dd.p, 2 * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(phase, dp.p, (size_t)n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (kernel_ms) *kernel_ms = ms;
    if (e != cudaSuccess) return jerr(g, BSG_ERR_CUDA, std::string("bsg_jumpgen_sort1: ") + cudaGetErrorString(e));
    return BSG_OK;
}

}  // extern "C"
