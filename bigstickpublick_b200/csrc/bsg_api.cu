// C ABI entry points: create / destroy / applyH / stats / errors, the
// host-side table validator and the derivation of the row layouts.
//
// bsg_create receives the reference's module arrays (bsg.h), validates every
// index before anything touches the GPU (the reference's own checks are
// check_opbundle_bounds, src/bparallel_opbundles.f90:1232-1286, and the
// sortedness check of src/bsortjumpslib.f90:228-241), uploads the arrays
// unchanged, and derives the output-stationary row layout in separate
// buffers.  It replaces getLoadDist / set_bundledXY_threadstart
// (src/bapplyhlibOMP.f90:34-868, src/bsortjumpslib.f90:491-713): instead of
// per-thread output ranges, each output row gets the list of contributions
// that land in it.

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <new>
#include <numeric>
#include <set>
#include <thread>
#include <unordered_map>

#include "bsg_internal.h"

namespace bsg {

int set_err(bsg_ctx *ctx, int code, const std::string &msg) {
    if (ctx) {
        ctx->last_error = msg;
        ctx->last_status = code;
    }
    return code;
}

int cuda_check(bsg_ctx *ctx, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return BSG_OK;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return set_err(ctx, BSG_ERR_NOMEM, std::string(what) + ": " + cudaGetErrorString(e));
    }
    return set_err(ctx, BSG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int dev_alloc(bsg_ctx *ctx, DevBuf &b, size_t bytes) {
    dev_free(b);
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        b.p = nullptr;
        return cuda_check(ctx, e, "cudaMalloc");
    }
    b.bytes = bytes;
    return BSG_OK;
}

void dev_free(DevBuf &b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

int upload(bsg_ctx *ctx, DevBuf &b, const void *src, size_t bytes) {
    int st = dev_alloc(ctx, b, bytes);
    if (st) return st;
    if (bytes && src) return cuda_check(ctx, cudaMemcpy(b.p, src, bytes, cudaMemcpyHostToDevice), "upload");
    return BSG_OK;
}

void build_tile_list(const bsg_ctx *ctx, int tp, std::vector<Tile> &tiles) {
    // tiles of tp positions, heaviest rows first (longest-processing-time order)
    std::vector<int32_t> order(ctx->nrows);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t x, int32_t y) { return ctx->h_work[x] > ctx->h_work[y]; });
    tiles.clear();
    for (int32_t r : order)
        for (int32_t p0 = 0; p0 < ctx->h_rowlen[r]; p0 += tp) {
            Tile t;
            t.row = r;
            t.pos0 = p0;
            t.npos = std::min(tp, ctx->h_rowlen[r] - p0);
            t.pad = 0;
            tiles.push_back(t);
        }
}

const TileSet *get_tiles(bsg_ctx *ctx, int tp) {
    auto it = ctx->tiles.find(tp);
    if (it != ctx->tiles.end()) return &it->second;
    std::vector<Tile> tiles;
    build_tile_list(ctx, tp, tiles);
    TileSet ts;
    if (upload(ctx, ts.buf, tiles.data(), tiles.size() * sizeof(Tile))) return nullptr;
    ts.ntiles = (int32_t)tiles.size();
    auto res = ctx->tiles.emplace(tp, ts);
    return &res.first->second;
}

}  // namespace bsg

using namespace bsg;

namespace {

// fn(i) for every i in [0, n), on up to 32 host threads taking chunks of
// `chunk` indices from a shared counter.  Callers write only to locations
// that index i owns, so the result does not depend on the schedule.
// max_threads 1 runs inline: small systems (and the many systems of a batch,
// which are already set up on parallel host threads) skip the thread start-up.
template <typename F>
void parallel_for(int64_t n, int64_t chunk, F fn, int max_threads = 32) {
    const int64_t nchunks = (n + chunk - 1) / chunk;
    const unsigned hw = std::max(1u, std::min((unsigned)std::max(1, max_threads), std::thread::hardware_concurrency()));
    const int nt = (int)std::min<int64_t>((int64_t)hw, nchunks);
    if (nt <= 1) {
        for (int64_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<int64_t> next{0};
    std::atomic<bool> oom{false};
    auto work = [&]() {
        try {
            for (;;) {
                const int64_t c = next.fetch_add(1);
                if (c >= nchunks || oom) return;
                const int64_t i1 = std::min(n, (c + 1) * chunk);
                for (int64_t i = c * chunk; i < i1; ++i) fn(i);
            }
        } catch (const std::bad_alloc &) {
            oom = true;   // reported to the caller below as an allocation failure
        }
    };
    std::vector<std::thread> th;
    for (int k = 1; k < nt; ++k) th.emplace_back(work);
    work();
    for (auto &x : th) x.join();
    if (oom) throw std::bad_alloc();
}
// f() on its own host thread; join() waits and reports an allocation failure
struct Task {
    std::thread th;
    bool oom = false;
    template <typename F>
    explicit Task(F f) : th([this, f]() {
        try {
            f();
        } catch (const std::bad_alloc &) {
            oom = true;
        }
    }) {}
    bool join() {
        th.join();
        return !oom;
    }
};

struct Validator {
    bsg_ctx *ctx;
    std::string msg;
    int fail(const std::string &m) {
        msg = m;
        return BSG_ERR_BAD_TABLE;
    }
};

template <typename T>
bool nonnull(const T *p, int64_t n) { return n == 0 || p != nullptr; }

// CSR by output position, stable (table order inside a position)
template <typename Rec>
void csr_by_out(const std::vector<int32_t> &out, const std::vector<Rec> &recs, int32_t nout,
                std::vector<int32_t> &ptr, std::vector<Rec> &sorted) {
    ptr.assign(nout + 1, 0);
    for (int32_t o : out) ptr[o + 1]++;
    for (int32_t i = 0; i < nout; ++i) ptr[i + 1] += ptr[i];
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    sorted.resize(recs.size());
    for (size_t k = 0; k < recs.size(); ++k) sorted[fill[out[k]]++] = recs[k];
}

// t3: the three-body arrays (bsg_create3), or null for a two-body context
int derive(bsg_ctx *ctx, const bsg_tables *t, const bsg_tables3 *t3, bool do_upload = true) {
    Validator V{ctx, ""};
    const bool three = (t3 != nullptr);
    ctx->threebody = three;
    // host threads for the derivation only where it is worth their start-up
    const int nthr = t->dimbasis >= (int64_t)1 << 20 ? 32 : 1;
    // ---- basic presence and sizes
    if (t->dimbasis <= 0 || t->nsd_p <= 0 || t->nsd_n <= 0)
        return set_err(ctx, BSG_ERR_BAD_TABLE, "empty basis");
    if (!t->pstart || !t->nstart) return set_err(ctx, BSG_ERR_BAD_TABLE, "pstart/nstart missing");
    // a three-body run labels its two-body jumps by pairs (t3 cop/dop), not by p2b_op/n2b_op
    if (!nonnull(t->p1b_isd, t->np1b) || !nonnull(t->p1b_fsd, t->np1b) || !nonnull(t->p1b_cop, t->np1b) ||
        !nonnull(t->p1b_dop, t->np1b) || !nonnull(t->p1b_phase, t->np1b) || !nonnull(t->n1b_isd, t->nn1b) ||
        !nonnull(t->n1b_fsd, t->nn1b) || !nonnull(t->n1b_cop, t->nn1b) || !nonnull(t->n1b_dop, t->nn1b) ||
        !nonnull(t->n1b_phase, t->nn1b) || !nonnull(t->p2b_isd, t->np2b) || !nonnull(t->p2b_fsd, t->np2b) ||
        (!three && !nonnull(t->p2b_op, t->np2b)) || !nonnull(t->p2b_phase, t->np2b) ||
        !nonnull(t->n2b_isd, t->nn2b) || !nonnull(t->n2b_fsd, t->nn2b) || (!three && !nonnull(t->n2b_op, t->nn2b)) ||
        !nonnull(t->n2b_phase, t->nn2b) || !nonnull(t->hmatpp, t->nmatpp) || !nonnull(t->hmatnn, t->nmatnn) ||
        !nonnull(t->hmatpn, t->nmatpn))
        return set_err(ctx, BSG_ERR_BAD_TABLE, "a table with nonzero length has a null pointer");
    if (three) {
        if (!nonnull(t3->p2b_cop, t->np2b) || !nonnull(t3->p2b_dop, t->np2b) || !nonnull(t3->n2b_cop, t->nn2b) ||
            !nonnull(t3->n2b_dop, t->nn2b) || t3->np3b < 0 || t3->nn3b < 0 || !nonnull(t3->p3b_isd, t3->np3b) ||
            !nonnull(t3->p3b_fsd, t3->np3b) || !nonnull(t3->p3b_op, t3->np3b) || !nonnull(t3->p3b_phase, t3->np3b) ||
            !nonnull(t3->n3b_isd, t3->nn3b) || !nonnull(t3->n3b_fsd, t3->nn3b) || !nonnull(t3->n3b_op, t3->nn3b) ||
            !nonnull(t3->n3b_phase, t3->nn3b) || t3->nmatppp < 0 || t3->nmatnnn < 0 || t3->nmatppn < 0 ||
            t3->nmatpnn < 0 || !nonnull(t3->hmatppp, t3->nmatppp) || !nonnull(t3->hmatnnn, t3->nmatnnn) ||
            !nonnull(t3->hmatppn, t3->nmatppn) || !nonnull(t3->hmatpnn, t3->nmatpnn) || t3->npairs_p < 0 ||
            t3->npairs_n < 0 || t3->npairs_p > 65535 || t3->npairs_n > 65535)
            return set_err(ctx, BSG_ERR_BAD_TABLE, "a three-body table with nonzero length has a null pointer, or a bad size");
        if ((t3->nmatppn > 0 && (!t3->cppntriplet || !t3->dppntriplet)) ||
            (t3->nmatpnn > 0 && (!t3->cpnntriplet || !t3->dpnntriplet)))
            return set_err(ctx, BSG_ERR_BAD_TABLE, "cppntriplet/dppntriplet or cpnntriplet/dpnntriplet missing");
        if (t->nmatpn + t3->nmatppn + t3->nmatpnn >= INT32_MAX || t->nmatnn + t3->nmatnnn >= INT32_MAX)
            return set_err(ctx, BSG_ERR_UNSUPPORTED, "three-body tables beyond this build's index widths");
    }
    if (t->nbundles < 0 || (t->nbundles > 0 && (!t->optype || !t->hchar || !t->pxstart || !t->pxend ||
                                                 !t->nxstart || !t->nxend || !t->cstride)))
        return set_err(ctx, BSG_ERR_BAD_TABLE, "opbundle arrays missing");
    if (t->dimbasis > (int64_t)INT32_MAX * 8 || t->nsd_p > INT32_MAX || t->nmatpn >= INT32_MAX)
        return set_err(ctx, BSG_ERR_UNSUPPORTED, "table sizes beyond this build's index widths");

    // ---- rows (proton SDs): pstart strictly increasing, row lengths
    const int64_t nrows = t->nsd_p;
    ctx->nrows = nrows;
    ctx->h_rowlen.assign(nrows, 0);
    if (t->pstart[0] != 0) return set_err(ctx, BSG_ERR_BAD_TABLE, "pstart(1) must be 0");
    for (int64_t p = 0; p < nrows; ++p) {
        const int64_t end = (p + 1 < nrows) ? t->pstart[p + 1] : t->dimbasis;
        const int64_t len = end - t->pstart[p];
        if (len <= 0 || len > INT32_MAX / 2)
            return set_err(ctx, BSG_ERR_BAD_TABLE, "pstart not strictly increasing at proton SD " + std::to_string(p + 1));
        ctx->h_rowlen[p] = (int32_t)len;
    }
    ctx->max_rowlen = *std::max_element(ctx->h_rowlen.begin(), ctx->h_rowlen.end());
    {
        std::vector<int32_t> tmp(ctx->h_rowlen);
        std::nth_element(tmp.begin(), tmp.begin() + tmp.size() / 2, tmp.end());
        ctx->median_rowlen = tmp[tmp.size() / 2];
    }
    for (int64_t n = 0; n < t->nsd_n; ++n)
        if (t->nstart[n] < 1 || t->nstart[n] > ctx->max_rowlen)
            return set_err(ctx, BSG_ERR_OOB_INDEX, "nstart out of range at neutron SD " + std::to_string(n + 1));
    std::unordered_map<int64_t, int32_t> row_of;
    row_of.reserve(nrows * 2);
    for (int64_t p = 0; p < nrows; ++p) row_of[t->pstart[p]] = (int32_t)p;
    auto rowof = [&](int64_t pst, int32_t &r) -> bool {
        auto it = row_of.find(pst);
        if (it == row_of.end()) return false;
        r = it->second;
        return true;
    };
    // the rows of every proton jump's isd and fsd, looked up once (bundles
    // share the jumps; -1: not a pstart value, reported where it is used)
    auto jump_rows = [&](const int64_t *isd, const int64_t *fsd, int64_t n, std::vector<int32_t> &ri,
                         std::vector<int32_t> &rf) {
        ri.assign((size_t)std::max<int64_t>(n, 0), -1);
        rf.assign((size_t)std::max<int64_t>(n, 0), -1);
        if (n <= 0 || !isd || !fsd) return;
        parallel_for(n, 1 << 14, [&](int64_t x) {
            int32_t r;
            if (rowof(isd[x], r)) ri[x] = r;
            if (rowof(fsd[x], r)) rf[x] = r;
        }, nthr);
    };
    std::vector<int32_t> p1b_ri, p1b_rf, p2b_ri, p2b_rf, p3b_ri, p3b_rf;
    jump_rows(t->p1b_isd, t->p1b_fsd, t->np1b, p1b_ri, p1b_rf);
    jump_rows(t->p2b_isd, t->p2b_fsd, t->np2b, p2b_ri, p2b_rf);
    if (t3) jump_rows(t3->p3b_isd, t3->p3b_fsd, t3->np3b, p3b_ri, p3b_rf);

    const int nl_n = t->nhsps_nl, nr_n = t->nhsps_nr, nl_p = t->nhsps_pl, nr_p = t->nhsps_pr;
    if (nl_n < 0 || nr_n < 0 || nl_p < 0 || nr_p < 0 || nl_n + nr_n > 250)
        return set_err(ctx, BSG_ERR_BAD_TABLE, "bad nhsps bounds");
    const int32_t ld = nl_n + nr_n + 1;
    const int64_t ncpn = (int64_t)ld * (nl_p + nr_p + 1);
    if (t->nmatpn > 0 && (!t->cpnpair || !t->dpnpair)) return set_err(ctx, BSG_ERR_BAD_TABLE, "cpnpair/dpnpair missing");
    std::vector<int32_t> cpn32(ncpn, 0), dpn32(ncpn, 0);
    if (t->cpnpair)
        for (int64_t i = 0; i < ncpn; ++i) {
            if (t->cpnpair[i] < 0 || t->cpnpair[i] > t->nmatpn || t->dpnpair[i] < 0 || t->dpnpair[i] > t->nmatpn)
                return set_err(ctx, BSG_ERR_OOB_INDEX, "cpnpair/dpnpair entry outside hmatpn");
            cpn32[i] = (int32_t)t->cpnpair[i];
            dpn32[i] = (int32_t)t->dpnpair[i];
        }
    // three-body PPN / PNN tables appended to the PN ones, so that the PN
    // machinery addresses all three: one table (cpn, dpn) and one matrix
    // element array hmatpn | hmatppn | hmatpnn.  The c entries carry the
    // matrix-element offset of their block; each combination is checked
    // against its own block when a bundle uses it.
    //   PPN block (base_ppn): (a + nhsps(-2)) + (bb - 1) * ld, a neutron s.p.
    //     label, bb a proton pair -- one column per proton pair, the rows the
    //     neutron labels the PN machinery tabulates;
    //   PNN block (base_pnn): (bb - 1) + (a + nhsps(-1)) * npairs_n, as the
    //     reference's cpnntriplet(bb, a).
    const int64_t npp3 = three ? t3->npairs_p : 0, nnp3 = three ? t3->npairs_n : 0;
    const int32_t ld_p = nl_p + nr_p + 1;
    const int64_t base_ppn = ncpn, base_pnn = ncpn + (int64_t)ld * npp3;
    const int64_t ncpn_all = base_pnn + nnp3 * ld_p;
    const int64_t off_ppn = t->nmatpn, off_pnn = t->nmatpn + (three ? t3->nmatppn : 0);
    if (ncpn_all >= INT32_MAX) return set_err(ctx, BSG_ERR_UNSUPPORTED, "triplet tables beyond this build's index widths");
    // raw (reference-layout) PPN / PNN entries for the per-bundle checks
    auto ppn_c = [&](int bb, int a) { return t3->cppntriplet[(int64_t)(bb - 1) + (int64_t)(a + nl_n) * npp3]; };
    auto ppn_d = [&](int dd, int c) { return t3->dppntriplet[(int64_t)(dd - 1) + (int64_t)(c + nl_n) * npp3]; };
    auto pnn_c = [&](int bb, int a) { return t3->cpnntriplet[(int64_t)(bb - 1) + (int64_t)(a + nl_p) * nnp3]; };
    auto pnn_d = [&](int dd, int c) { return t3->dpnntriplet[(int64_t)(dd - 1) + (int64_t)(c + nl_p) * nnp3]; };
    if (three) {
        cpn32.resize(ncpn_all, 0);
        dpn32.resize(ncpn_all, 0);
        if (t3->nmatppn > 0)
            for (int bb = 1; bb <= npp3; ++bb)
                for (int a = -nl_n; a <= nr_n; ++a) {
                    const int64_t at = base_ppn + (a + nl_n) + (int64_t)(bb - 1) * ld;
                    cpn32[at] = ppn_c(bb, a) + (int32_t)off_ppn;
                    dpn32[at] = ppn_d(bb, a);
                }
        if (t3->nmatpnn > 0)
            for (int a = -nl_p; a <= nr_p; ++a)
                for (int bb = 1; bb <= nnp3; ++bb) {
                    const int64_t at = base_pnn + (bb - 1) + (int64_t)(a + nl_p) * nnp3;
                    cpn32[at] = pnn_c(bb, a) + (int32_t)off_pnn;
                    dpn32[at] = pnn_d(bb, a);
                }
    }

    // ---- neutron operators
    struct NKey {
        int kind, dir;
        int64_t x0, x1;
        bool operator<(const NKey &o) const {
            return std::tie(kind, dir, x0, x1) < std::tie(o.kind, o.dir, o.x0, o.x1);
        }
    };
    std::map<NKey, int32_t> nop_id;
    std::vector<NOp> nops;
    std::vector<int32_t> nop_maxin;
    std::vector<int32_t> nptr_all;
    std::vector<PNRec> pnrec_all;
    std::vector<NNRec> nnrec_all;
    std::vector<int32_t> nnrec_op_all;
    std::vector<int8_t> nnrec_ph_all;
    std::vector<BDPair> bd_all;
    // neutron operators of a sector jump's jump range, by source:
    //   0 NN  (n2b, hmatnn label records -> matrix-element records)
    //   1 PN  (n1b, s.p. labels b, d -> label records)
    //   2 PNN (n2b with pair labels bb, dd -> label records)
    //   3 NNN (n3b, hmatnnn label records -> matrix-element records)
    // Matrix-element records keep their label for the adjoint and for the
    // 32-bit records; NNN labels are offset by nmatnn (one device array
    // hmatnn | hmatnnn).
    std::vector<int32_t> nop_nsub;         // label operators: sub-operators from this id on (0: a later one)
    std::vector<int32_t> nop_nbd;          // label operators: pairs over all sub-operators
    std::vector<int32_t> bdk_dense;        // (b,d) -> index in the op's list, reset after each op
    std::vector<size_t> bdk_touched;
    auto get_nop = [&](int kind, int dir, int64_t x0, int64_t x1, int32_t &id) -> int {
        NKey k{kind, dir, x0, x1};
        auto it = nop_id.find(k);
        if (it != nop_id.end()) { id = it->second; return BSG_OK; }
        const int64_t n = x1 - x0 + 1;
        std::vector<int32_t> out(n);
        int32_t maxin = -1, maxout = -1;
        NOp op{};
        op.kind = (kind == 1 || kind == 2) ? 1 : 0;
        if (op.kind == 1) {
            const bool pnn = (kind == 2);
            const int64_t nkey = pnn ? nnp3 : ld;   // labels per side
            if (bdk_dense.size() < (size_t)(nkey * nkey)) bdk_dense.assign((size_t)(nkey * nkey), -1);
            std::vector<PNRec> recs(n);
            std::vector<BDPair> bdl;
            for (int64_t x = x0; x <= x1; ++x) {
                const int64_t isd = pnn ? t->n2b_isd[x - 1] : t->n1b_isd[x - 1];
                const int64_t fsd = pnn ? t->n2b_fsd[x - 1] : t->n1b_fsd[x - 1];
                if (isd < 1 || fsd < 1 || isd > ctx->max_rowlen || fsd > ctx->max_rowlen)
                    return V.fail(std::string(pnn ? "n2b" : "n1b") + " isd/fsd out of range at jump " + std::to_string(x));
                int kb, kd;   // row keys into the cpn / dpn tables
                if (pnn) {
                    const int bb = t3->n2b_cop[x - 1], dd = t3->n2b_dop[x - 1];
                    if (bb < 1 || bb > nnp3 || dd < 1 || dd > nnp3)
                        return V.fail("n2b_cop/dop outside the neutron pairs at jump " + std::to_string(x));
                    kb = bb - 1;
                    kd = dd - 1;
                } else {
                    const int b = t->n1b_cop[x - 1], d = t->n1b_dop[x - 1];
                    if (b < -nl_n || b > nr_n || d < -nl_n || d > nr_n || b == 0 || d == 0)
                        return V.fail("n1b_cop/dop outside the neutron half spaces at jump " + std::to_string(x));
                    kb = b + nl_n;
                    kd = d + nl_n;
                }
                const int ph = pnn ? t->n2b_phase[x - 1] : t->n1b_phase[x - 1];
                if (ph != 1 && ph != -1) return V.fail(pnn ? "n2b_phase not +-1" : "n1b_phase not +-1");
                const size_t key = (size_t)kb * nkey + kd;
                int32_t &kk = bdk_dense[key];
                if (kk < 0) {
                    kk = (int32_t)bdl.size();
                    bdk_touched.push_back(key);
                    bdl.push_back(BDPair{(uint16_t)kb, (uint16_t)kd});
                }
                PNRec r;
                r.in = (int32_t)((dir == 0 ? isd : fsd) - 1);
                out[x - x0] = (int32_t)((dir == 0 ? fsd : isd) - 1);
                r.k = (uint16_t)kk;
                r.ph = (int8_t)ph;
                r.pad = 0;
                recs[x - x0] = r;
                maxin = std::max(maxin, r.in);
                maxout = std::max(maxout, out[x - x0]);
                if (bdl.size() > 65535) break;
            }
            for (size_t key : bdk_touched) bdk_dense[key] = -1;
            bdk_touched.clear();
            if (bdl.size() > 65535) return V.fail("too many distinct (b,d) label pairs in a neutron sector jump");
            // more label pairs than one shared table holds: consecutive
            // sub-operators over slices of the pair list, each with the
            // records whose pair falls in its slice (same output positions,
            // record order kept); a contribution on the operator becomes one
            // contribution per sub-operator
            const int32_t tmax = std::max<int32_t>(32, ctx->pn_table_max);
            const int32_t nbd_all = (int32_t)bdl.size();
            const int32_t nsub = std::max<int32_t>(1, (nbd_all + tmax - 1) / tmax);
            const int32_t bd0 = (int32_t)bd_all.size();
            bd_all.insert(bd_all.end(), bdl.begin(), bdl.end());
            id = (int32_t)nops.size();
            for (int32_t sb = 0; sb < nsub; ++sb) {
                const int32_t k0 = sb * tmax, k1 = std::min(nbd_all, k0 + tmax);
                std::vector<int32_t> sout;
                std::vector<PNRec> srec;
                if (nsub == 1) {
                    sout.swap(out);
                    srec.swap(recs);
                } else {
                    for (int64_t x = 0; x < n; ++x)
                        if (recs[x].k >= k0 && recs[x].k < k1) {
                            PNRec r = recs[x];
                            r.k = (uint16_t)(r.k - k0);
                            srec.push_back(r);
                            sout.push_back(out[x]);
                        }
                }
                std::vector<int32_t> ptr;
                std::vector<PNRec> sorted;
                csr_by_out(sout, srec, maxout + 1, ptr, sorted);
                NOp so = op;
                so.rec_base = (int64_t)pnrec_all.size();
                so.ptr_base = (int64_t)nptr_all.size();
                so.nout = maxout + 1;
                so.bd_base = bd0 + k0;
                so.nbd = k1 - k0;
                pnrec_all.insert(pnrec_all.end(), sorted.begin(), sorted.end());
                nptr_all.insert(nptr_all.end(), ptr.begin(), ptr.end());
                nops.push_back(so);
                nop_maxin.push_back(maxin);
                nop_nsub.push_back(sb == 0 ? nsub : 0);
                nop_nbd.push_back(sb == 0 ? nbd_all : 0);
            }
            nop_id[k] = id;
            return BSG_OK;
        } else {
            const bool nnn = (kind == 3);
            const int64_t *xisd = nnn ? t3->n3b_isd : t->n2b_isd, *xfsd = nnn ? t3->n3b_fsd : t->n2b_fsd;
            const int32_t *xop = nnn ? t3->n3b_op : t->n2b_op;
            const int8_t *xph = nnn ? t3->n3b_phase : t->n2b_phase;
            const float *hm = nnn ? t3->hmatnnn : t->hmatnn;
            const int64_t nmat = nnn ? t3->nmatnnn : t->nmatnn;
            const int32_t loff = nnn ? (int32_t)t->nmatnn : 0;
            const char *nm = nnn ? "n3b" : "n2b";
            std::vector<NNRec> recs(n);
            std::vector<int32_t> ops(n);
            std::vector<int8_t> phs(n);
            for (int64_t x = x0; x <= x1; ++x) {
                const int64_t isd = xisd[x - 1], fsd = xfsd[x - 1];
                if (isd < 1 || fsd < 1 || isd > ctx->max_rowlen || fsd > ctx->max_rowlen)
                    return V.fail(std::string(nm) + " isd/fsd out of range at jump " + std::to_string(x));
                const int32_t opl = xop[x - 1];
                if (opl < 1 || opl > nmat)
                    return V.fail(std::string(nm) + (nnn ? "_op outside hmatnnn" : "_op outside hmatnn") + " at jump " +
                                  std::to_string(x));
                const int ph = xph[x - 1];
                if (ph != 1 && ph != -1) return V.fail(std::string(nm) + "_phase not +-1");
                NNRec r;
                r.in = (int32_t)((dir == 0 ? isd : fsd) - 1);
                out[x - x0] = (int32_t)((dir == 0 ? fsd : isd) - 1);
                float xme = hm[opl - 1];
                xme = xme * (float)ph;
                r.me = xme;
                recs[x - x0] = r;
                ops[x - x0] = opl + loff;
                phs[x - x0] = (int8_t)ph;
                maxin = std::max(maxin, r.in);
                maxout = std::max(maxout, out[x - x0]);
            }
            std::vector<int32_t> ptr;
            std::vector<NNRec> sorted;
            csr_by_out(out, recs, maxout + 1, ptr, sorted);
            std::vector<int32_t> sorted_ops;
            csr_by_out(out, ops, maxout + 1, ptr, sorted_ops);
            std::vector<int8_t> sorted_phs;
            csr_by_out(out, phs, maxout + 1, ptr, sorted_phs);
            nnrec_ph_all.insert(nnrec_ph_all.end(), sorted_phs.begin(), sorted_phs.end());
            op.rec_base = (int64_t)nnrec_all.size();
            op.ptr_base = (int64_t)nptr_all.size();
            op.nout = maxout + 1;
            nnrec_all.insert(nnrec_all.end(), sorted.begin(), sorted.end());
            nnrec_op_all.insert(nnrec_op_all.end(), sorted_ops.begin(), sorted_ops.end());
            nptr_all.insert(nptr_all.end(), ptr.begin(), ptr.end());
        }
        id = (int32_t)nops.size();
        nops.push_back(op);
        nop_maxin.push_back(maxin);
        nop_nsub.push_back(1);
        nop_nbd.push_back(0);
        nop_id[k] = id;
        return BSG_OK;
    };

    // ---- contributions per row
    std::vector<std::pair<int32_t, PPContrib>> pp;
    std::vector<int32_t> pp_op_tmp;
    std::vector<int8_t> pp_ph_tmp;
    std::vector<std::pair<int32_t, NNContrib>> nn;
    std::vector<std::pair<int32_t, PNContrib>> pn;
    std::vector<std::pair<int32_t, SPEContrib>> spe;
    int64_t ops[4] = {0, 0, 0, 0};
    int64_t ops3[4] = {0, 0, 0, 0};   // PPP, NNN, PPN, PNN
    struct PPBundle { int64_t ib, px0, px1, nx0, nx1; bool bwd; };
    std::vector<PPBundle> pp_bundles;
    // one proton-side PN-form contribution (PN, PPN, PNN) of the jump s1 -> s2
    auto pn_contrib = [&](int64_t s1, int32_t ri, int32_t rf, int32_t id, int32_t aoff, int32_t coff, int ph,
                          const std::string &what) -> int {
        if (ri < 0 || rf < 0) return set_err(ctx, BSG_ERR_OOB_INDEX, what + " isd/fsd is not a pstart value");
        if (nops[id].nout > ctx->h_rowlen[rf] || nop_maxin[id] >= ctx->h_rowlen[ri])
            return set_err(ctx, BSG_ERR_OOB_INDEX, what + ": neutron jump outside the row");
        if (ph != 1 && ph != -1) return set_err(ctx, BSG_ERR_BAD_TABLE, what + " phase not +-1");
        for (int32_t sb = 0; sb < nop_nsub[id]; ++sb) {
            PNContrib c{};
            c.q_off = s1;
            c.nop = id + sb;
            c.aoff = aoff;
            c.coff = coff;
            c.php = (float)ph;
            pn.push_back({rf, c});
        }
        return BSG_OK;
    };
    {
        // one PN-form contribution per proton jump and neutron sub-operator:
        // room for one per jump up front (most operators have one part), so
        // the vector is not copied over and over while it grows
        int64_t npn = 0, nnn = 0, nspe = 0;
        for (int64_t ib = 0; ib < t->nbundles; ++ib) {
            const int op = t->optype[ib];
            const int64_t n = std::max<int64_t>(0, t->pxend[ib] - t->pxstart[ib] + 1);
            if (op == BSG_OP_PN || op == BSG_OP_PPN || op == BSG_OP_PNN) npn += n;
            else if (op == BSG_OP_NN || op == BSG_OP_NNN) nnn += n;
            else if (op == BSG_OP_SPE) nspe += n;
        }
        pn.reserve((size_t)npn);
        nn.reserve((size_t)nnn);
        spe.reserve((size_t)nspe);
    }
    for (int64_t ib = 0; ib < t->nbundles; ++ib) {
        const int op = t->optype[ib], hc = t->hchar[ib];
        const int64_t px0 = t->pxstart[ib], px1 = t->pxend[ib], nx0 = t->nxstart[ib], nx1 = t->nxend[ib];
        const int64_t cs = t->cstride[ib];
        const std::string where = " (opbundle " + std::to_string(ib + 1) + ")";
        if (hc != 'f' && hc != 'b' && hc != 'h') return set_err(ctx, BSG_ERR_BAD_TABLE, "bad hchar" + where);
        if (cs < 1) return set_err(ctx, BSG_ERR_BAD_TABLE, "cstride < 1" + where);
        if (px1 < px0 || nx1 < nx0) continue;  // empty bundle: no work
        const bool bwd = (hc == 'b');
        const bool is3 = (op == BSG_OP_PPP || op == BSG_OP_NNN || op == BSG_OP_PPN || op == BSG_OP_PNN);
        if (is3 && !three) return set_err(ctx, BSG_ERR_BAD_TABLE, "three-body bundle in a two-body context" + where);
        // applyHbundled_g with threebody set applies SPE and the three-body
        // bundles only (src/bapplyhlib1.f90:107-235)
        if (three && (op == BSG_OP_PP || op == BSG_OP_NN || op == BSG_OP_PN)) continue;
        if (op == BSG_OP_PPP) {
            // applyhPPPbundled_g (src/bapplyhlib1.f90:1390-1572): as PP
            if (px0 < 1 || px1 > t3->np3b || nx0 < 1 || nx1 > t->nsd_n)
                return set_err(ctx, BSG_ERR_OOB_INDEX, "PPP range" + where);
            if (cs != 1) return set_err(ctx, BSG_ERR_UNSUPPORTED, "PPP cstride != 1" + where);
            for (int64_t c = nx0 + 1; c <= nx1; ++c)
                if (t->nstart[c - 1] != t->nstart[c - 2] + 1)
                    return set_err(ctx, BSG_ERR_UNSUPPORTED, "PPP neutron run not contiguous" + where);
            const int32_t lo = (int32_t)(t->nstart[nx0 - 1] - 1), hi = (int32_t)(t->nstart[nx1 - 1] - 1);
            for (int64_t x = px0; x <= px1; ++x) {
                const int64_t s1 = bwd ? t3->p3b_fsd[x - 1] : t3->p3b_isd[x - 1];
                const int32_t ri = bwd ? p3b_rf[x - 1] : p3b_ri[x - 1], rf = bwd ? p3b_ri[x - 1] : p3b_rf[x - 1];
                if (ri < 0 || rf < 0)
                    return set_err(ctx, BSG_ERR_OOB_INDEX, "p3b isd/fsd is not a pstart value" + where);
                if (hi >= ctx->h_rowlen[ri] || hi >= ctx->h_rowlen[rf])
                    return set_err(ctx, BSG_ERR_OOB_INDEX, "PPP neutron run longer than the row" + where);
                const int32_t opl = t3->p3b_op[x - 1];
                if (opl < 1 || opl > t3->nmatppp) return set_err(ctx, BSG_ERR_OOB_INDEX, "p3b_op outside hmatppp" + where);
                const int ph = t3->p3b_phase[x - 1];
                if (ph != 1 && ph != -1) return set_err(ctx, BSG_ERR_BAD_TABLE, "p3b_phase not +-1" + where);
                PPContrib c{};
                c.q_off = s1;
                float xme = t3->hmatppp[opl - 1];
                xme = xme * (float)ph;
                c.me = xme;
                c.lo = lo;
                c.hi = hi;
                pp.push_back({rf, c});
                pp_op_tmp.push_back(opl);
                pp_ph_tmp.push_back((int8_t)ph);
            }
            ops3[0] += (px1 - px0 + 1) * (nx1 - nx0 + 1);
            continue;
        }
        if (op == BSG_OP_NNN) {
            // applyhNNNbundled_g (src/bapplyhlib1.f90:1579-1756): as NN
            if (px0 < 1 || px1 > t->nsd_p || nx0 < 1 || nx1 > t3->nn3b)
                return set_err(ctx, BSG_ERR_OOB_INDEX, "NNN range" + where);
            int32_t id;
            int st = get_nop(3, bwd ? 1 : 0, nx0, nx1, id);
            if (st) return set_err(ctx, st, V.msg + where);
            int64_t nrow_b = 0;
            for (int64_t csd = px0; csd <= px1; csd += cs) {
                const int32_t r = (int32_t)(csd - 1);
                if (nops[id].nout > ctx->h_rowlen[r] || nop_maxin[id] >= ctx->h_rowlen[r])
                    return set_err(ctx, BSG_ERR_OOB_INDEX, "NNN jump outside the row" + where);
                nn.push_back({r, NNContrib{id}});
                ++nrow_b;
            }
            ops3[1] += nrow_b * (nx1 - nx0 + 1);
            continue;
        }
        if (op == BSG_OP_PPN || op == BSG_OP_PNN) {
            // applyhPPNbundled_g / applyhPNNbundled_g (src/bapplyhlib1.f90:2295-2562,
            // :2033-2285): PN-form contributions on the appended tables
            const bool ppn = (op == BSG_OP_PPN);
            const char *nm = ppn ? "PPN" : "PNN";
            if (ppn ? (px0 < 1 || px1 > t->np2b || nx0 < 1 || nx1 > t->nn1b)
                    : (px0 < 1 || px1 > t->np1b || nx0 < 1 || nx1 > t->nn2b))
                return set_err(ctx, BSG_ERR_OOB_INDEX, std::string(nm) + " range" + where);
            if ((ppn && t3->nmatppn == 0) || (!ppn && t3->nmatpnn == 0))
                return set_err(ctx, BSG_ERR_BAD_TABLE, std::string(nm) + " bundle without matrix elements" + where);
            int32_t id;
            int st = get_nop(ppn ? 1 : 2, bwd ? 1 : 0, nx0, nx1, id);
            if (st) return set_err(ctx, st, V.msg + where);
            // every proton (created, destroyed) label pair x neutron (b,d) pair
            // of the bundle must address its own matrix-element block
            const NOp &no = nops[id];
            std::vector<std::pair<int, int>> lab;
            {
                std::set<std::pair<int, int>> seen;
                for (int64_t x = px0; x <= px1; ++x) {
                    int cl, dl;
                    if (ppn) {
                        cl = t3->p2b_cop[x - 1];
                        dl = t3->p2b_dop[x - 1];
                        if (cl < 1 || cl > npp3 || dl < 1 || dl > npp3)
                            return set_err(ctx, BSG_ERR_OOB_INDEX, "p2b_cop/dop outside the proton pairs" + where);
                    } else {
                        cl = t->p1b_cop[x - 1];
                        dl = t->p1b_dop[x - 1];
                        if (cl < -nl_p || cl > nr_p || dl < -nl_p || dl > nr_p || cl == 0 || dl == 0)
                            return set_err(ctx, BSG_ERR_OOB_INDEX, "p1b_cop/dop outside the proton half spaces" + where);
                    }
                    if (seen.insert({cl, dl}).second) lab.push_back({cl, dl});
                }
            }
            const int64_t nmat3 = ppn ? t3->nmatppn : t3->nmatpnn;
            for (auto &pl : lab)
                for (int32_t k = 0; k < nop_nbd[id]; ++k) {
                    const BDPair bd = bd_all[no.bd_base + k];
                    const int64_t idx = ppn ? (int64_t)ppn_c(pl.first, bd.b - nl_n) + ppn_d(pl.second, bd.d - nl_n)
                                            : (int64_t)pnn_c(bd.b + 1, pl.first) + pnn_d(bd.d + 1, pl.second);
                    if (idx < 1 || idx > nmat3)
                        return set_err(ctx, BSG_ERR_OOB_INDEX,
                                       std::string(ppn ? "cppntriplet+dppntriplet outside hmatppn" : "cpnntriplet+dpnntriplet outside hmatpnn") + where);
                }
            for (int64_t x = px0; x <= px1; ++x) {
                int64_t isd, fsd;
                int32_t risd, rfsd;
                int cl, dl, ph;
                int32_t aoff, coff;
                if (ppn) {
                    isd = t->p2b_isd[x - 1];
                    fsd = t->p2b_fsd[x - 1];
                    risd = p2b_ri[x - 1];
                    rfsd = p2b_rf[x - 1];
                    cl = t3->p2b_cop[x - 1];
                    dl = t3->p2b_dop[x - 1];
                    ph = t->p2b_phase[x - 1];
                    aoff = (int32_t)(base_ppn + (int64_t)(cl - 1) * ld);
                    coff = (int32_t)(base_ppn + (int64_t)(dl - 1) * ld);
                } else {
                    isd = t->p1b_isd[x - 1];
                    fsd = t->p1b_fsd[x - 1];
                    risd = p1b_ri[x - 1];
                    rfsd = p1b_rf[x - 1];
                    cl = t->p1b_cop[x - 1];
                    dl = t->p1b_dop[x - 1];
                    ph = t->p1b_phase[x - 1];
                    aoff = (int32_t)(base_pnn + (int64_t)(cl + nl_p) * nnp3);
                    coff = (int32_t)(base_pnn + (int64_t)(dl + nl_p) * nnp3);
                }
                st = pn_contrib(bwd ? fsd : isd, bwd ? rfsd : risd, bwd ? risd : rfsd, id, aoff, coff, ph,
                                std::string(nm) + where);
                if (st) return st;
            }
            ops3[ppn ? 2 : 3] += (px1 - px0 + 1) * (nx1 - nx0 + 1);
            continue;
        }
        if (op == BSG_OP_PP) {
            if (px0 < 1 || px1 > t->np2b || nx0 < 1 || nx1 > t->nsd_n)
                return set_err(ctx, BSG_ERR_OOB_INDEX, "PP range" + where);
            if (cs != 1) return set_err(ctx, BSG_ERR_UNSUPPORTED, "PP cstride != 1" + where);
            for (int64_t c = nx0 + 1; c <= nx1; ++c)
                if (t->nstart[c - 1] != t->nstart[c - 2] + 1)
                    return set_err(ctx, BSG_ERR_UNSUPPORTED, "PP neutron run not contiguous" + where);
            // the jumps are checked and turned into contributions after the
            // loop, all PP bundles at once on host threads (PP contributions
            // only go to `pp`, which keeps the bundle order)
            pp_bundles.push_back({ib, px0, px1, nx0, nx1, bwd});
            ops[1] += (px1 - px0 + 1) * (nx1 - nx0 + 1);
        } else if (op == BSG_OP_NN) {
            if (px0 < 1 || px1 > t->nsd_p || nx0 < 1 || nx1 > t->nn2b)
                return set_err(ctx, BSG_ERR_OOB_INDEX, "NN range" + where);
            int32_t id;
            int st = get_nop(0, bwd ? 1 : 0, nx0, nx1, id);
            if (st) return set_err(ctx, st, V.msg + where);
            int64_t nrow_b = 0;
            for (int64_t csd = px0; csd <= px1; csd += cs) {
                const int32_t r = (int32_t)(csd - 1);
                if (nops[id].nout > ctx->h_rowlen[r] || nop_maxin[id] >= ctx->h_rowlen[r])
                    return set_err(ctx, BSG_ERR_OOB_INDEX, "NN jump outside the row" + where);
                NNContrib c{id};
                nn.push_back({r, c});
                ++nrow_b;
            }
            ops[2] += nrow_b * (nx1 - nx0 + 1);
        } else if (op == BSG_OP_PN) {
            if (px0 < 1 || px1 > t->np1b || nx0 < 1 || nx1 > t->nn1b)
                return set_err(ctx, BSG_ERR_OOB_INDEX, "PN range" + where);
            int32_t id;
            int st = get_nop(1, bwd ? 1 : 0, nx0, nx1, id);
            if (st) return set_err(ctx, st, V.msg + where);
            // every (a,c) x (b,d) combination of the bundle must address hmatpn
            std::vector<std::pair<int, int>> ac, bd;
            {
                std::vector<char> seen((size_t)(nl_p + nr_p + 1) * (nl_p + nr_p + 1), 0);
                for (int64_t x = px0; x <= px1; ++x) {
                    const int a = t->p1b_cop[x - 1], c = t->p1b_dop[x - 1];
                    if (a < -nl_p || a > nr_p || c < -nl_p || c > nr_p || a == 0 || c == 0)
                        return set_err(ctx, BSG_ERR_OOB_INDEX, "p1b_cop/dop outside the proton half spaces" + where);
                    char &s = seen[(size_t)(a + nl_p) * (nl_p + nr_p + 1) + (c + nl_p)];
                    if (!s) { s = 1; ac.push_back({a, c}); }
                }
                std::vector<char> seen2((size_t)ld * ld, 0);
                for (int64_t x = nx0; x <= nx1; ++x) {
                    const int b = t->n1b_cop[x - 1], d = t->n1b_dop[x - 1];
                    char &s = seen2[(size_t)(b + nl_n) * ld + (d + nl_n)];
                    if (!s) { s = 1; bd.push_back({b, d}); }
                }
                for (auto &p1 : ac)
                    for (auto &p2 : bd) {
                        const int64_t i1 = (int64_t)(p2.first + nl_n) + (int64_t)(p1.first + nl_p) * ld;
                        const int64_t i2 = (int64_t)(p2.second + nl_n) + (int64_t)(p1.second + nl_p) * ld;
                        const int64_t idx = t->cpnpair[i1] + t->dpnpair[i2];
                        if (idx < 1 || idx > t->nmatpn)
                            return set_err(ctx, BSG_ERR_OOB_INDEX, "cpnpair+dpnpair outside hmatpn" + where);
                    }
            }
            for (int64_t x = px0; x <= px1; ++x) {
                const int64_t s1 = bwd ? t->p1b_fsd[x - 1] : t->p1b_isd[x - 1];
                const int32_t ri = bwd ? p1b_rf[x - 1] : p1b_ri[x - 1], rf = bwd ? p1b_ri[x - 1] : p1b_rf[x - 1];
                if (ri < 0 || rf < 0)
                    return set_err(ctx, BSG_ERR_OOB_INDEX, "p1b isd/fsd is not a pstart value" + where);
                if (nops[id].nout > ctx->h_rowlen[rf] || nop_maxin[id] >= ctx->h_rowlen[ri])
                    return set_err(ctx, BSG_ERR_OOB_INDEX, "PN neutron jump outside the row" + where);
                const int ph = t->p1b_phase[x - 1];
                if (ph != 1 && ph != -1) return set_err(ctx, BSG_ERR_BAD_TABLE, "p1b_phase not +-1" + where);
                for (int32_t sb = 0; sb < nop_nsub[id]; ++sb) {
                    PNContrib c{};
                    c.q_off = s1;
                    c.nop = id + sb;
                    c.aoff = (int32_t)(t->p1b_cop[x - 1] + nl_p) * ld;
                    c.coff = (int32_t)(t->p1b_dop[x - 1] + nl_p) * ld;
                    c.php = (float)ph;
                    pn.push_back({rf, c});
                }
            }
            ops[3] += (px1 - px0 + 1) * (nx1 - nx0 + 1);
        } else if (op == BSG_OP_SPE) {
            if (!t->call_spe || !t->pspe_h || !t->nspe_h)
                return set_err(ctx, BSG_ERR_BAD_TABLE, "SPE bundle without pspe_h/nspe_h" + where);
            if (px0 < 1 || px1 > t->nsd_p || nx0 < 1 || nx1 > t->nsd_n)
                return set_err(ctx, BSG_ERR_OOB_INDEX, "SPE range" + where);
            for (int64_t ip = px0; ip <= px1; ++ip) {
                SPEContrib c{};
                c.pspe = t->pspe_h[ip - 1];
                c.lo = (int32_t)(t->nstart[nx0 - 1] - 1);
                c.hi = c.lo + (int32_t)(nx1 - nx0);
                c.n0 = (int32_t)(nx0 - 1);
                if (c.hi >= ctx->h_rowlen[ip - 1])
                    return set_err(ctx, BSG_ERR_OOB_INDEX, "SPE run longer than the row" + where);
                spe.push_back({(int32_t)(ip - 1), c});
            }
            ops[0] += (px1 - px0 + 1) * (nx1 - nx0 + 1);
        } else {
            return set_err(ctx, BSG_ERR_BAD_TABLE, "unknown optype" + where);
        }
    }
    if (!pp_bundles.empty()) {
        // PP bundles (src/bapplyhlibOMP.f90:1068-1241), one per task; the
        // first failing bundle in table order reports
        // one contribution per jump: every bundle writes its own slice
        const size_t nb_pp = pp_bundles.size();
        std::vector<size_t> at0(nb_pp + 1, pp.size());
        for (size_t j = 0; j < nb_pp; ++j) at0[j + 1] = at0[j] + (size_t)(pp_bundles[j].px1 - pp_bundles[j].px0 + 1);
        pp.resize(at0[nb_pp]);
        pp_op_tmp.resize(at0[nb_pp]);
        pp_ph_tmp.resize(at0[nb_pp]);
        std::vector<int> bst(nb_pp, BSG_OK);
        std::vector<std::string> bmsg(nb_pp);
        parallel_for((int64_t)nb_pp, 1, [&](int64_t j) {
            const PPBundle &B = pp_bundles[j];
            const int32_t lo = (int32_t)(t->nstart[B.nx0 - 1] - 1), hi = (int32_t)(t->nstart[B.nx1 - 1] - 1);
            auto fail = [&](int code, const char *m) {
                bst[j] = code;
                bmsg[j] = std::string(m) + " (opbundle " + std::to_string(B.ib + 1) + ")";
            };
            size_t at = at0[j];
            for (int64_t x = B.px0; x <= B.px1; ++x, ++at) {
                const int64_t s1 = B.bwd ? t->p2b_fsd[x - 1] : t->p2b_isd[x - 1];
                const int32_t ri = B.bwd ? p2b_rf[x - 1] : p2b_ri[x - 1], rf = B.bwd ? p2b_ri[x - 1] : p2b_rf[x - 1];
                if (ri < 0 || rf < 0) return fail(BSG_ERR_OOB_INDEX, "p2b isd/fsd is not a pstart value");
                if (hi >= ctx->h_rowlen[ri] || hi >= ctx->h_rowlen[rf])
                    return fail(BSG_ERR_OOB_INDEX, "PP neutron run longer than the row");
                const int32_t opl = t->p2b_op[x - 1];
                if (opl < 1 || opl > t->nmatpp) return fail(BSG_ERR_OOB_INDEX, "p2b_op outside hmatpp");
                const int ph = t->p2b_phase[x - 1];
                if (ph != 1 && ph != -1) return fail(BSG_ERR_BAD_TABLE, "p2b_phase not +-1");
                PPContrib c{};
                c.q_off = s1;
                float xme = t->hmatpp[opl - 1];
                xme = xme * (float)ph;
                c.me = xme;
                c.lo = lo;
                c.hi = hi;
                pp[at] = {rf, c};
                pp_op_tmp[at] = opl;
                pp_ph_tmp[at] = (int8_t)ph;
            }
        }, nthr);
        for (size_t j = 0; j < nb_pp; ++j)
            if (bst[j]) return set_err(ctx, bst[j], bmsg[j]);
    }
    ctx->stats.n_ops_spe = ops[0];
    ctx->stats.n_ops_pp = ops[1];
    ctx->stats.n_ops_nn = ops[2];
    ctx->stats.n_ops_pn = ops[3];
    ctx->stats.n_ops_ppp = ops3[0];
    ctx->stats.n_ops_nnn = ops3[1];
    ctx->stats.n_ops_ppn = ops3[2];
    ctx->stats.n_ops_pnn = ops3[3];

    // ---- assign each row's contributions to the kWarps warps of its CTA by
    // longest-processing-time (heaviest first to the least loaded warp), then
    // flatten into CSR over (row, warp) slots.  Inside a slot the bundle order
    // is kept (PN grouped by neutron operator for cache reuse).
    {
        // stable sort by (row, operator): a counting sort by row, then each
        // row's run stably by operator (rows in parallel)
        std::vector<int64_t> rs(nrows + 1, 0);
        for (auto &e : pn) rs[e.first + 1]++;
        for (int64_t r = 0; r < nrows; ++r) rs[r + 1] += rs[r];
        std::vector<std::pair<int32_t, PNContrib>> sorted(pn.size());
        {
            std::vector<int64_t> fill(rs.begin(), rs.end() - 1);
            for (auto &e : pn) sorted[fill[e.first]++] = e;
        }
        parallel_for(nrows, 256, [&](int64_t r) {
            std::stable_sort(sorted.begin() + rs[r], sorted.begin() + rs[r + 1],
                             [](const std::pair<int32_t, PNContrib> &x, const std::pair<int32_t, PNContrib> &y) {
                                 return x.second.nop < y.second.nop;
                             });
        }, nthr);
        pn.swap(sorted);
    }
    auto nrec_of = [&](int32_t id) -> int64_t { return nptr_all[nops[id].ptr_base + nops[id].nout]; };
    // ---- sliced records: per operator, output positions in slices of 32;
    // a slice holds its longest position's count of 32-record rows, record k
    // of lane l at row k (padding rows hold {0, 0} and are never read)
    std::vector<int2> sell_all;
    std::vector<int32_t> slice_off_all;
    // 32-bit copy when every input position, (b,d) index and hmatnn label fits
    int32_t max_nbd_all = 0;
    for (const NOp &op : nops) max_nbd_all = std::max(max_nbd_all, op.nbd);
    // PN records need the position and the (b,d) index to fit; NN records
    // carry the hmatnn label, which only the FP64 kernels read: when the
    // labels do not fit, the NN entries stay zero and FP64 keeps the 8-byte
    // records (ctx->rec32_nn)
    const int64_t nmatnn_all = t->nmatnn + (three ? t3->nmatnnn : 0);
    const bool pack32 = ctx->max_rowlen <= 65536 && max_nbd_all <= 32768;
    const bool nn32 = pack32 && nmatnn_all <= 32768;
    ctx->rec32_nn = nn32;
    std::vector<uint32_t> sell32_all;
    {
        // sizes per operator (parallel), offsets (in operator order), fill (parallel)
        const int64_t nop_all = (int64_t)nops.size();
        std::vector<int64_t> op_recs(nop_all, 0);
        std::atomic<bool> too_big{false};
        parallel_for(nop_all, 16, [&](int64_t o) {
            const NOp &op = nops[o];
            const int32_t *ptr = nptr_all.data() + op.ptr_base;
            int64_t off = 0;
            for (int sl = 0; sl < (op.nout + 31) / 32; ++sl) {
                int32_t width = 0;
                for (int l = 0; l < 32 && 32 * sl + l < op.nout; ++l)
                    width = std::max(width, ptr[32 * sl + l + 1] - ptr[32 * sl + l]);
                if (off > INT32_MAX) too_big = true;
                off += (int64_t)32 * width;
            }
            op_recs[o] = off;
        }, nthr);
        if (too_big) return V.fail("a neutron operator has more than 2^31 sliced records");
        int64_t nrec_tot = 0, nslice_tot = 0;
        for (int64_t o = 0; o < nop_all; ++o) {
            nops[o].sell_base = nrec_tot;
            nops[o].slice_base = nslice_tot;
            nrec_tot += op_recs[o];
            nslice_tot += (nops[o].nout + 31) / 32;
        }
        sell_all.assign((size_t)nrec_tot, make_int2(0, 0));   // padding rows hold {0, 0}
        if (pack32) sell32_all.assign((size_t)nrec_tot, 0u);
        slice_off_all.assign((size_t)nslice_tot, 0);
        parallel_for(nop_all, 16, [&](int64_t o) {
            const NOp &op = nops[o];
            const int32_t *ptr = nptr_all.data() + op.ptr_base;
            int64_t off = 0;
            for (int sl = 0; sl < (op.nout + 31) / 32; ++sl) {
                int32_t width = 0;
                for (int l = 0; l < 32 && 32 * sl + l < op.nout; ++l)
                    width = std::max(width, ptr[32 * sl + l + 1] - ptr[32 * sl + l]);
                slice_off_all[op.slice_base + sl] = (int32_t)off;
                const size_t row0 = (size_t)(op.sell_base + off);
                for (int l = 0; l < 32 && 32 * sl + l < op.nout; ++l)
                    for (int32_t k = ptr[32 * sl + l]; k < ptr[32 * sl + l + 1]; ++k) {
                        int2 r;
                        uint32_t r32;
                        if (op.kind == 1) {
                            const PNRec &pr = pnrec_all[op.rec_base + k];
                            std::memcpy(&r, &pr, sizeof(int2));
                            r32 = (uint32_t)pr.in | ((uint32_t)pr.k << 16) | (pr.ph < 0 ? 0x80000000u : 0u);
                        } else {
                            std::memcpy(&r, &nnrec_all[op.rec_base + k], sizeof(int2));
                            r32 = nn32 ? (uint32_t)nnrec_all[op.rec_base + k].in |
                                             ((uint32_t)(nnrec_op_all[op.rec_base + k] - 1) << 16) |
                                             (nnrec_ph_all[op.rec_base + k] < 0 ? 0x80000000u : 0u)
                                       : 0u;
                        }
                        const size_t at = row0 + (size_t)32 * (k - ptr[32 * sl + l]) + l;
                        sell_all[at] = r;
                        if (pack32) sell32_all[at] = r32;
                    }
                off += (int64_t)32 * width;
            }
        }, nthr);
    }
    const int W = kRowWarps;
    std::vector<uint8_t> w_pp(pp.size()), w_nn(nn.size()), w_pn(pn.size()), w_spe(spe.size());
    {
        struct Ref { int64_t wgt; int8_t type; int32_t idx; };
        std::vector<std::vector<int32_t>> by[4];
        for (int k = 0; k < 4; ++k) by[k].assign(0, {});
        std::vector<int32_t> cnt[4], start[4];
        auto bucket = [&](auto &v, int k) {
            cnt[k].assign(nrows + 1, 0);
            for (auto &e : v) cnt[k][e.first + 1]++;
            for (int64_t r = 0; r < nrows; ++r) cnt[k][r + 1] += cnt[k][r];
            start[k].assign(v.size(), 0);
            std::vector<int32_t> fill(cnt[k].begin(), cnt[k].end() - 1);
            for (size_t i = 0; i < v.size(); ++i) start[k][fill[v[i].first]++] = (int32_t)i;
        };
        bucket(pp, 0); bucket(nn, 1); bucket(pn, 2); bucket(spe, 3);
        // rows are independent: each writes only its own contributions' warps
        parallel_for(nrows, 256, [&](int64_t r) {
            thread_local std::vector<Ref> refs;
            refs.clear();
            for (int32_t q = cnt[0][r]; q < cnt[0][r + 1]; ++q) {
                const auto &c = pp[start[0][q]].second;
                refs.push_back({(int64_t)(c.hi - c.lo + 1), 0, start[0][q]});
            }
            for (int32_t q = cnt[1][r]; q < cnt[1][r + 1]; ++q)
                refs.push_back({nrec_of(nn[start[1][q]].second.nop) + 32, 1, start[1][q]});
            for (int32_t q = cnt[2][r]; q < cnt[2][r + 1]; ++q) {
                const int32_t id = pn[start[2][q]].second.nop;
                refs.push_back({nrec_of(id) + nops[id].nbd + 32, 2, start[2][q]});
            }
            for (int32_t q = cnt[3][r]; q < cnt[3][r + 1]; ++q) {
                const auto &c = spe[start[3][q]].second;
                refs.push_back({(int64_t)(c.hi - c.lo + 1), 3, start[3][q]});
            }
            std::stable_sort(refs.begin(), refs.end(), [](const Ref &x, const Ref &y) { return x.wgt > y.wgt; });
            int64_t load[kRowWarps] = {0};
            for (const Ref &f : refs) {
                int best = 0;
                for (int w = 1; w < W; ++w)
                    if (load[w] < load[best]) best = w;
                load[best] += f.wgt;
                (f.type == 0 ? w_pp : f.type == 1 ? w_nn : f.type == 2 ? w_pn : w_spe)[f.idx] = (uint8_t)best;
            }
        }, nthr);
    }
    // CSR over (row, warp) slots; inside a slot the contributions keep their
    // order (a counting sort by slot, stable in the input order)
    auto by_slot = [&](auto &v, const std::vector<uint8_t> &wv, std::vector<int32_t> &ptr, auto &flat,
                       std::vector<int32_t> *perm) {
        const int64_t nslot = nrows * W;
        std::vector<int64_t> key(v.size());
        parallel_for((int64_t)v.size(), 1 << 16, [&](int64_t i) { key[i] = (int64_t)v[i].first * W + wv[i]; }, nthr);
        ptr.assign(nslot + 1, 0);
        for (int64_t k : key) ptr[k + 1]++;
        for (int64_t r = 0; r < nslot; ++r) ptr[r + 1] += ptr[r];
        std::vector<size_t> idx(v.size());
        {
            std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
            for (size_t i = 0; i < v.size(); ++i) idx[fill[key[i]]++] = i;
        }
        flat.resize(v.size());
        if (perm) perm->resize(v.size());
        parallel_for((int64_t)idx.size(), 1 << 16, [&](int64_t k) {
            flat[k] = v[idx[k]].second;
            if (perm) (*perm)[k] = (int32_t)idx[k];
        }, nthr);
    };
    if (pp.size() > (size_t)INT32_MAX || pn.size() > (size_t)INT32_MAX)
        return set_err(ctx, BSG_ERR_UNSUPPORTED, "more than 2^31 row contributions");
    std::vector<int32_t> spe_ptr, pp_perm;
    std::vector<SPEContrib> h_spe;
    if (nthr == 1) {
        by_slot(pp, w_pp, ctx->h_pp_ptr, ctx->h_pp, &pp_perm);
        by_slot(nn, w_nn, ctx->h_nn_ptr, ctx->h_nn, nullptr);
        by_slot(pn, w_pn, ctx->h_pn_ptr, ctx->h_pn, nullptr);
        by_slot(spe, w_spe, spe_ptr, h_spe, nullptr);
    } else {
        // the four slot layouts are independent
        Task tnn([&]() { by_slot(nn, w_nn, ctx->h_nn_ptr, ctx->h_nn, nullptr); });
        Task tpn([&]() { by_slot(pn, w_pn, ctx->h_pn_ptr, ctx->h_pn, nullptr); });
        Task tspe([&]() { by_slot(spe, w_spe, spe_ptr, h_spe, nullptr); });
        bool ok = true;
        try {
            by_slot(pp, w_pp, ctx->h_pp_ptr, ctx->h_pp, &pp_perm);
        } catch (const std::bad_alloc &) {
            ok = false;
        }
        ok = tnn.join() && ok;
        ok = tpn.join() && ok;
        ok = tspe.join() && ok;
        if (!ok) throw std::bad_alloc();
    }
    ctx->h_pp_op.resize(pp_perm.size());
    ctx->h_pp_ph.resize(pp_perm.size());
    for (size_t k = 0; k < pp_perm.size(); ++k) {
        ctx->h_pp_op[k] = pp_op_tmp[pp_perm[k]];
        ctx->h_pp_ph[k] = pp_ph_tmp[pp_perm[k]];
    }
    ctx->h_nops = nops;
    ctx->h_nnrec_op = nnrec_op_all;

    // per-row work estimate (operations) for tile ordering
    ctx->h_work.assign(nrows, 0);
    for (int64_t r = 0; r < nrows; ++r) {
        int64_t w = 0;
        for (int32_t c = ctx->h_pp_ptr[r * W]; c < ctx->h_pp_ptr[(r + 1) * W]; ++c) w += ctx->h_pp[c].hi - ctx->h_pp[c].lo + 1;
        for (int32_t c = ctx->h_nn_ptr[r * W]; c < ctx->h_nn_ptr[(r + 1) * W]; ++c) w += nrec_of(ctx->h_nn[c].nop);
        for (int32_t c = ctx->h_pn_ptr[r * W]; c < ctx->h_pn_ptr[(r + 1) * W]; ++c) w += nrec_of(ctx->h_pn[c].nop);
        ctx->h_work[r] = (int32_t)std::min<int64_t>(w, INT32_MAX);
    }

    if (!do_upload) return BSG_OK;
    // ---- upload: raw tables (unchanged) and derived layouts
    auto up = [&](DevBuf &b, const void *src, size_t bytes) { return upload(ctx, b, src, bytes); };
    int st = 0;
    std::vector<int64_t> row_off(t->pstart, t->pstart + nrows);
    const void *raw_ptrs[] = {t->pstart, t->nstart, t->p1b_isd, t->p1b_fsd, t->p1b_cop, t->p1b_dop, t->p1b_phase,
                              t->n1b_isd, t->n1b_fsd, t->n1b_cop, t->n1b_dop, t->n1b_phase,
                              t->p2b_isd, t->p2b_fsd, t->p2b_op, t->p2b_phase,
                              t->n2b_isd, t->n2b_fsd, t->n2b_op, t->n2b_phase,
                              t->hmatpp, t->hmatnn, t->cpnpair, t->dpnpair};
    const size_t raw_bytes[] = {8 * (size_t)t->nsd_p, 8 * (size_t)t->nsd_n, 8 * (size_t)t->np1b, 8 * (size_t)t->np1b,
                                2 * (size_t)t->np1b, 2 * (size_t)t->np1b, (size_t)t->np1b,
                                8 * (size_t)t->nn1b, 8 * (size_t)t->nn1b, 2 * (size_t)t->nn1b, 2 * (size_t)t->nn1b, (size_t)t->nn1b,
                                8 * (size_t)t->np2b, 8 * (size_t)t->np2b, 4 * (size_t)t->np2b, (size_t)t->np2b,
                                8 * (size_t)t->nn2b, 8 * (size_t)t->nn2b, 4 * (size_t)t->nn2b, (size_t)t->nn2b,
                                4 * (size_t)t->nmatpp, 4 * (size_t)t->nmatnn,
                                t->cpnpair ? 8 * (size_t)ncpn : 0, t->dpnpair ? 8 * (size_t)ncpn : 0};
    std::vector<const void *> rp(raw_ptrs, raw_ptrs + sizeof(raw_ptrs) / sizeof(raw_ptrs[0]));
    std::vector<size_t> rb(raw_bytes, raw_bytes + sizeof(raw_bytes) / sizeof(raw_bytes[0]));
    if (three) {
        const void *p3[] = {t3->p2b_cop, t3->p2b_dop, t3->n2b_cop, t3->n2b_dop, t3->p3b_isd, t3->p3b_fsd, t3->p3b_op,
                            t3->p3b_phase, t3->n3b_isd, t3->n3b_fsd, t3->n3b_op, t3->n3b_phase, t3->hmatppp,
                            t3->hmatnnn, t3->cppntriplet, t3->dppntriplet, t3->cpnntriplet, t3->dpnntriplet};
        const size_t nt_p = (size_t)npp3 * ld, nt_n = (size_t)nnp3 * ld_p;
        const size_t b3[] = {4 * (size_t)t->np2b, 4 * (size_t)t->np2b, 4 * (size_t)t->nn2b, 4 * (size_t)t->nn2b,
                             8 * (size_t)t3->np3b, 8 * (size_t)t3->np3b, 4 * (size_t)t3->np3b, (size_t)t3->np3b,
                             8 * (size_t)t3->nn3b, 8 * (size_t)t3->nn3b, 4 * (size_t)t3->nn3b, (size_t)t3->nn3b,
                             4 * (size_t)t3->nmatppp, 4 * (size_t)t3->nmatnnn, 4 * nt_p, 4 * nt_p, 4 * nt_n, 4 * nt_n};
        rp.insert(rp.end(), p3, p3 + sizeof(p3) / sizeof(p3[0]));
        rb.insert(rb.end(), b3, b3 + sizeof(b3) / sizeof(b3[0]));
    }
    const int nraw = (int)rb.size();
    ctx->raw.resize(nraw);
    int64_t jb = 0;
    for (int i = 0; i < nraw && !st; ++i) {
        const size_t bytes = rp[i] ? rb[i] : 0;   // an unused table (e.g. p2b_op of a three-body run)
        st = up(ctx->raw[i], rp[i], bytes);
        jb += (int64_t)bytes;
    }
    if (st) return st;
    ctx->stats.jump_bytes = jb;
    // hmatpn doubles as raw table and kernel operand; a three-body context
    // appends hmatppn and hmatpnn (the PPN / PNN blocks of the cpn table)
    {
        std::vector<float> hpn(t->hmatpn ? t->hmatpn : nullptr, t->hmatpn ? t->hmatpn + t->nmatpn : nullptr);
        if (three) {
            if (t3->nmatppn) hpn.insert(hpn.end(), t3->hmatppn, t3->hmatppn + t3->nmatppn);
            if (t3->nmatpnn) hpn.insert(hpn.end(), t3->hmatpnn, t3->hmatpnn + t3->nmatpnn);
        }
        if ((st = up(ctx->hmatpn, hpn.data(), 4 * hpn.size()))) return st;
        ctx->stats.jump_bytes += 4 * (int64_t)hpn.size();
    }
    std::vector<float> hnn_all(t->hmatnn ? t->hmatnn : nullptr, t->hmatnn ? t->hmatnn + t->nmatnn : nullptr);
    if (three && t3->nmatnnn) hnn_all.insert(hnn_all.end(), t3->hmatnnn, t3->hmatnnn + t3->nmatnnn);
    std::vector<float> nspe(t->nsd_n, 0.0f);
    if (t->call_spe && t->nspe_h) std::copy(t->nspe_h, t->nspe_h + t->nsd_n, nspe.begin());
    if ((st = up(ctx->row_off, row_off.data(), 8 * row_off.size())) ||
        (st = up(ctx->pp_ptr, ctx->h_pp_ptr.data(), 4 * ctx->h_pp_ptr.size())) ||
        (st = up(ctx->nn_ptr, ctx->h_nn_ptr.data(), 4 * ctx->h_nn_ptr.size())) ||
        (st = up(ctx->pn_ptr, ctx->h_pn_ptr.data(), 4 * ctx->h_pn_ptr.size())) ||
        (st = up(ctx->spe_ptr, spe_ptr.data(), 4 * spe_ptr.size())) ||
        (st = up(ctx->pp, ctx->h_pp.data(), sizeof(PPContrib) * ctx->h_pp.size())) ||
        (st = up(ctx->nn, ctx->h_nn.data(), sizeof(NNContrib) * ctx->h_nn.size())) ||
        (st = up(ctx->pn, ctx->h_pn.data(), sizeof(PNContrib) * ctx->h_pn.size())) ||
        (st = up(ctx->spe, h_spe.data(), sizeof(SPEContrib) * h_spe.size())) ||
        (st = up(ctx->nops, nops.data(), sizeof(NOp) * nops.size())) ||
        (st = up(ctx->nptr, nptr_all.data(), 4 * nptr_all.size())) ||
        (st = up(ctx->pnrec, pnrec_all.data(), sizeof(PNRec) * pnrec_all.size())) ||
        (st = up(ctx->nnrec, nnrec_all.data(), sizeof(NNRec) * nnrec_all.size())) ||
        (st = up(ctx->sell, sell_all.data(), sizeof(int2) * sell_all.size())) ||
        (pack32 && (st = up(ctx->sell32, sell32_all.data(), 4 * sell32_all.size()))) ||
        (st = up(ctx->slice_off, slice_off_all.data(), 4 * slice_off_all.size())) ||
        (st = up(ctx->bd, bd_all.data(), sizeof(BDPair) * bd_all.size())) ||
        (st = up(ctx->cpn, cpn32.data(), 4 * cpn32.size())) || (st = up(ctx->dpn, dpn32.data(), 4 * dpn32.size())) ||
        (st = up(ctx->nspe, nspe.data(), 4 * nspe.size())) ||
        (st = up(ctx->pp_op, ctx->h_pp_op.data(), 4 * ctx->h_pp_op.size())) ||
        (st = up(ctx->nnrec_op, nnrec_op_all.data(), 4 * nnrec_op_all.size())) ||
        (st = up(ctx->nnrec_ph, nnrec_ph_all.data(), nnrec_ph_all.size())) ||
        (st = up(ctx->pp_ph, ctx->h_pp_ph.data(), ctx->h_pp_ph.size())) ||
        (st = up(ctx->hmatpp_d, t->hmatpp, 4 * (size_t)t->nmatpp)) ||
        (st = up(ctx->hmatnn_d, hnn_all.data(), 4 * hnn_all.size())))
        return st;
    ctx->stats.derived_bytes = (int64_t)(8 * row_off.size() + 4 * (ctx->h_pp_ptr.size() * 3 + spe_ptr.size()) +
                                         sizeof(PPContrib) * ctx->h_pp.size() + sizeof(NNContrib) * ctx->h_nn.size() +
                                         sizeof(PNContrib) * ctx->h_pn.size() + sizeof(SPEContrib) * h_spe.size() +
                                         sizeof(NOp) * nops.size() + 4 * nptr_all.size() +
                                         sizeof(PNRec) * pnrec_all.size() + sizeof(NNRec) * nnrec_all.size() +
                                         sizeof(int2) * sell_all.size() + 4 * sell32_all.size() +
                                         4 * slice_off_all.size());
    ctx->stats.n_rows = nrows;
    ctx->stats.n_contrib = (int64_t)(ctx->h_pp.size() + ctx->h_nn.size() + ctx->h_pn.size() + h_spe.size());

    RowArgs &a = ctx->args;
    a.row_off = (const int64_t *)ctx->row_off.p;
    a.pp_ptr = (const int32_t *)ctx->pp_ptr.p;
    a.nn_ptr = (const int32_t *)ctx->nn_ptr.p;
    a.pn_ptr = (const int32_t *)ctx->pn_ptr.p;
    a.spe_ptr = (const int32_t *)ctx->spe_ptr.p;
    a.pp = (const PPContrib *)ctx->pp.p;
    a.nn = (const NNContrib *)ctx->nn.p;
    a.pn = (const PNContrib *)ctx->pn.p;
    a.spe = (const SPEContrib *)ctx->spe.p;
    a.nops = (const NOp *)ctx->nops.p;
    a.nptr = (const int32_t *)ctx->nptr.p;
    a.pnrec = (const PNRec *)ctx->pnrec.p;
    a.nnrec = (const NNRec *)ctx->nnrec.p;
    a.sell = (const int2 *)ctx->sell.p;
    a.sell32 = pack32 ? (const uint32_t *)ctx->sell32.p : nullptr;
    a.hmatnn = (const float *)ctx->hmatnn_d.p;
    a.slice_off = (const int32_t *)ctx->slice_off.p;
    a.bd = (const BDPair *)ctx->bd.p;
    int32_t max_nbd = 0;
    for (auto &o : nops) max_nbd = std::max(max_nbd, o.nbd);
    a.max_nbd = max_nbd;
    a.cols_out = nullptr;  // set per launch by the Lanczos path only
    a.cols_ld = 0;
    ctx->h_bd = bd_all;
    ctx->h_pnrec = pnrec_all;
    ctx->h_nptr = nptr_all;
    a.hmatpn = (const float *)ctx->hmatpn.p;
    a.cpn = (const int32_t *)ctx->cpn.p;
    a.dpn = (const int32_t *)ctx->dpn.p;
    a.nspe = (const float *)ctx->nspe.p;
    a.ld_cpn = ld;
    a.ncpn = (int32_t)cpn32.size();
    return BSG_OK;
}

void free_ctx(bsg_ctx *ctx) {
    for (auto &b : ctx->raw) dev_free(b);
    DevBuf *bufs[] = {&ctx->row_off, &ctx->pp_ptr, &ctx->nn_ptr, &ctx->pn_ptr, &ctx->spe_ptr, &ctx->pp, &ctx->nn,
                      &ctx->pn, &ctx->spe, &ctx->nops, &ctx->nptr, &ctx->pnrec, &ctx->nnrec, &ctx->bd, &ctx->sell,
                      &ctx->sell32, &ctx->slice_off, &ctx->hmatpn,
                      &ctx->cpn, &ctx->dpn, &ctx->nspe, &ctx->pp_op, &ctx->nnrec_op, &ctx->nnrec_ph, &ctx->pp_ph,
                      &ctx->hmatpp_d,
                      &ctx->hmatnn_d, &ctx->scratch_in, &ctx->scratch_out};
    for (DevBuf *b : bufs) dev_free(*b);
    for (auto &kv : ctx->tiles) dev_free(kv.second.buf);
    ctx->tiles.clear();
    for (auto &kv : ctx->chunk_tiles) dev_free(kv.second.buf);
    ctx->chunk_tiles.clear();
    for (cudaEvent_t e : ctx->chunk_ev) cudaEventDestroy(e);
    ctx->chunk_ev.clear();
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    ctx->copy_stream = nullptr;
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    ctx->ev0 = ctx->ev1 = nullptr;
    ctx->stream = nullptr;
}

}  // namespace

extern "C" {

const char *bsg_strerror(int status) {
    switch (status) {
    case BSG_OK: return "ok";
    case BSG_ERR_BAD_TABLE: return "table failed validation";
    case BSG_ERR_OOB_INDEX: return "index outside its array";
    case BSG_ERR_CUDA: return "CUDA error";
    case BSG_ERR_NOMEM: return "out of memory";
    case BSG_ERR_TIMEOUT: return "bounded device wait timed out";
    case BSG_ERR_NAN: return "non-finite value";
    case BSG_ERR_ARG: return "bad argument";
    case BSG_ERR_UNSUPPORTED: return "unsupported input";
    case BSG_ERR_NOT_CONVERGED: return "not converged";
    default: return "unknown status";
    }
}

int bsg_last_error(const bsg_ctx *ctx, char *buf, size_t len) {
    if (!ctx || !buf || len == 0) return BSG_ERR_ARG;
    std::snprintf(buf, len, "%s", ctx->last_error.c_str());
    return BSG_OK;
}

}  // extern "C"

namespace {
int create_ctx(const bsg_tables *t, const bsg_tables3 *t3, const bsg_config *cfg, bsg_ctx **out) {
    if (!out) return BSG_ERR_ARG;
    *out = nullptr;
    if (!t) return BSG_ERR_ARG;
    bsg_ctx *ctx = new (std::nothrow) bsg_ctx();
    if (!ctx) return BSG_ERR_NOMEM;
    ctx->device = cfg ? cfg->device : 0;
    ctx->max_nb = (cfg && cfg->max_nb > 0) ? cfg->max_nb : 16;
    // default split size, measured best on B200: 512 pairs for two-body PN
    // (no pf operator has more than 441), 384 for three-body runs (pf 4p4n:
    // 43.0 ms against 48.7 at 512, 45.3 at 256, 134.6 unsplit)
    ctx->pn_table_max = (cfg && cfg->pn_table_max > 0) ? cfg->pn_table_max : (t3 ? 384 : 512);
    int st = cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (!st) st = cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
    if (!st) st = cuda_check(ctx, cudaEventCreate(&ctx->ev0), "event");
    if (!st) st = cuda_check(ctx, cudaEventCreate(&ctx->ev1), "event");
    if (!st) {
        ctx->t = *t;
        ctx->dim = t->dimbasis;
        try {
            st = derive(ctx, t, t3);
        } catch (const std::bad_alloc &) {
            st = set_err(ctx, BSG_ERR_NOMEM, "host allocation failed while deriving row layouts");
        }
    }
    if (st) {
        std::fprintf(stderr, "bsg_create: %s: %s\n", bsg_strerror(st), ctx->last_error.c_str());
        free_ctx(ctx);
        delete ctx;
        return st;
    }
    ctx->stats.kernel_launches_per_matvec = 1;
    *out = ctx;
    return BSG_OK;
}
}  // namespace

extern "C" {

int bsg_create(const bsg_tables *t, const bsg_config *cfg, bsg_ctx **out) { return create_ctx(t, nullptr, cfg, out); }

int bsg_create3(const bsg_tables *t, const bsg_tables3 *t3, const bsg_config *cfg, bsg_ctx **out) {
    if (!t3) {
        if (out) *out = nullptr;
        return BSG_ERR_ARG;
    }
    return create_ctx(t, t3, cfg, out);
}

int bsg_validate_tables(const bsg_tables *t, char *msg, size_t len) { return bsg_validate_tables3(t, nullptr, msg, len); }

int bsg_validate_tables3(const bsg_tables *t, const bsg_tables3 *t3, char *msg, size_t len) {
    if (msg && len) msg[0] = 0;
    if (!t) return BSG_ERR_ARG;
    bsg_ctx *ctx = new (std::nothrow) bsg_ctx();
    if (!ctx) return BSG_ERR_NOMEM;
    ctx->t = *t;
    ctx->dim = t->dimbasis;
    int st;
    try {
        st = derive(ctx, t, t3, false);
    } catch (const std::bad_alloc &) {
        st = set_err(ctx, BSG_ERR_NOMEM, "host allocation failed while validating");
    }
    if (msg && len) std::snprintf(msg, len, "%s", ctx->last_error.c_str());
    delete ctx;
    return st;
}

int bsg_destroy(bsg_ctx *ctx) {
    if (!ctx) return BSG_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_ctx(ctx);
    delete ctx;
    return BSG_OK;
}

namespace {

// host-pointer applyH in kChunks row-range chunks when the output is at least
// kChunkBytes: each chunk's states are final when its launch ends, so their
// copy back overlaps the launches after it
constexpr int kChunks = 4;
constexpr size_t kChunkBytes = (size_t)32 << 20;

// the chunked tiles of width tp: rows cut into kChunks contiguous ranges of
// about equal estimated work, each range's tiles heaviest row first
const ChunkTiles *get_chunk_tiles(bsg_ctx *ctx, int tp) {
    auto it = ctx->chunk_tiles.find(tp);
    if (it != ctx->chunk_tiles.end()) return &it->second;
    ChunkTiles ct;
    int64_t total = 0;
    for (int32_t r = 0; r < ctx->nrows; ++r) total += ctx->h_work[r];
    std::vector<int32_t> rcut(1, 0);
    int64_t acc = 0;
    for (int32_t r = 0; r < ctx->nrows && (int)rcut.size() < kChunks; ++r) {
        acc += ctx->h_work[r];
        if (acc * kChunks >= total * (int64_t)rcut.size()) rcut.push_back(r + 1);
    }
    while ((int)rcut.size() <= kChunks) rcut.push_back(ctx->nrows);
    rcut.back() = ctx->nrows;
    std::vector<Tile> tiles;
    int64_t state = 0;
    for (int c = 0; c < kChunks; ++c) {
        std::vector<int32_t> order;
        for (int32_t r = rcut[c]; r < rcut[c + 1]; ++r) order.push_back(r);
        std::stable_sort(order.begin(), order.end(),
                         [&](int32_t x, int32_t y) { return ctx->h_work[x] > ctx->h_work[y]; });
        ct.start.push_back((int32_t)tiles.size());
        ct.s0.push_back(state);
        for (int32_t r : order)
            for (int32_t p0 = 0; p0 < ctx->h_rowlen[r]; p0 += tp) {
                Tile t;
                t.row = r;
                t.pos0 = p0;
                t.npos = std::min(tp, ctx->h_rowlen[r] - p0);
                t.pad = 0;
                tiles.push_back(t);
            }
        for (int32_t r = rcut[c]; r < rcut[c + 1]; ++r) state += ctx->h_rowlen[r];
    }
    ct.start.push_back((int32_t)tiles.size());
    ct.s0.push_back(state);
    if (upload(ctx, ct.buf, tiles.data(), tiles.size() * sizeof(Tile))) return nullptr;
    for (int c = 0; c < kChunks; ++c) {
        TileSet v;
        v.buf.p = (char *)ct.buf.p + (size_t)ct.start[c] * sizeof(Tile);
        v.buf.bytes = (size_t)(ct.start[c + 1] - ct.start[c]) * sizeof(Tile);
        v.ntiles = ct.start[c + 1] - ct.start[c];
        ct.view.push_back(v);
    }
    auto res = ctx->chunk_tiles.emplace(tp, std::move(ct));
    return &res.first->second;
}

// the chunk the next launch covers (the lookup has no other argument)
thread_local int t_chunk = 0;
const TileSet *chunk_lookup(bsg_ctx *ctx, int tp) {
    const ChunkTiles *ct = get_chunk_tiles(ctx, tp);
    return ct ? &ct->view[t_chunk] : nullptr;
}

// states of chunk c for the launch's tile width: every tile width cuts the
// rows the same way (the cut depends on the rows only), so any cached entry
// gives the ranges
const ChunkTiles *any_chunk_tiles(bsg_ctx *ctx) {
    return ctx->chunk_tiles.empty() ? nullptr : &ctx->chunk_tiles.begin()->second;
}

int applyh_on(bsg_ctx *ctx, const void *vin, void *vout, int nb, int prec, int flags, cudaStream_t s) {
    if (!vin || !vout || nb < 1 || nb > 64 || (prec != BSG_PREC_FP32 && prec != BSG_PREC_FP64))
        return set_err(ctx, BSG_ERR_ARG, "bsg_applyh: bad arguments");
    if (vin == vout) return set_err(ctx, BSG_ERR_ARG, "bsg_applyh: vin and vout must not alias");
    int st = cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (st) return st;
    const int acc = (flags & BSG_ACCUMULATE) ? 1 : 0;
    if (flags & BSG_DEVICE_PTRS) return launch_applyh(ctx, vin, vout, nb, prec, acc, s);
    // host pointers: copy in, apply, copy out (the drop-in path for vec1/vec2)
    const size_t bytes = (size_t)ctx->dim * nb * (prec == BSG_PREC_FP32 ? 4 : 8);
    if (ctx->scratch_in.bytes < bytes) {
        if ((st = dev_alloc(ctx, ctx->scratch_in, bytes)) || (st = dev_alloc(ctx, ctx->scratch_out, bytes))) return st;
    }
    st = cuda_check(ctx, cudaMemcpyAsync(ctx->scratch_in.p, vin, bytes, cudaMemcpyHostToDevice, s), "H2D vin");
    if (!st && acc) st = cuda_check(ctx, cudaMemcpyAsync(ctx->scratch_out.p, vout, bytes, cudaMemcpyHostToDevice, s), "H2D vout");
    if (st) return st;
    if (bytes < kChunkBytes || ctx->nrows < kChunks) {
        st = launch_applyh(ctx, ctx->scratch_in.p, ctx->scratch_out.p, nb, prec, acc, s);
        if (!st) st = cuda_check(ctx, cudaMemcpyAsync(vout, ctx->scratch_out.p, bytes, cudaMemcpyDeviceToHost, s), "D2H vout");
        if (!st) st = cuda_check(ctx, cudaStreamSynchronize(s), "applyh sync");
        return st;
    }
    // chunked: all launches queued first (each followed by its event), then
    // each chunk's copy on the copy stream after its event, so the copies
    // overlap the later launches whether vout is pinned or not
    if (!ctx->copy_stream &&
        (st = cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "copy stream")))
        return st;
    while ((int)ctx->chunk_ev.size() < kChunks) {
        cudaEvent_t e = nullptr;
        if ((st = cuda_check(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "chunk event"))) return st;
        ctx->chunk_ev.push_back(e);
    }
    for (int c = 0; c < kChunks && !st; ++c) {
        t_chunk = c;
        st = launch_applyh(ctx, ctx->scratch_in.p, ctx->scratch_out.p, nb, prec, acc, s, chunk_lookup);
        if (!st) st = cuda_check(ctx, cudaEventRecord(ctx->chunk_ev[c], s), "chunk event record");
    }
    t_chunk = 0;
    const ChunkTiles *ct = any_chunk_tiles(ctx);
    if (!st && !ct) st = set_err(ctx, BSG_ERR_NOMEM, "bsg_applyh: chunked row tiles");
    const size_t esz = (size_t)nb * (prec == BSG_PREC_FP32 ? 4 : 8);
    for (int c = 0; c < kChunks && !st; ++c) {
        const size_t off = (size_t)ct->s0[c] * esz, len = (size_t)(ct->s0[c + 1] - ct->s0[c]) * esz;
        st = cuda_check(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->chunk_ev[c], 0), "chunk wait");
        if (!st && len)
            st = cuda_check(ctx, cudaMemcpyAsync((char *)vout + off, (const char *)ctx->scratch_out.p + off, len,
                                                 cudaMemcpyDeviceToHost, ctx->copy_stream),
                            "D2H vout chunk");
    }
    // both streams drained before returning, also after an error
    const cudaError_t e1 = cudaStreamSynchronize(ctx->copy_stream), e2 = cudaStreamSynchronize(s);
    if (!st) st = cuda_check(ctx, e1 != cudaSuccess ? e1 : e2, "applyh sync");
    return st;
}

}  // namespace

// stream: the caller's cudaStream_t; NULL means the legacy default stream
int bsg_applyh_stream(bsg_ctx *ctx, const void *vin, void *vout, int nb, int prec, int flags, void *stream) {
    if (!ctx) return BSG_ERR_ARG;
    return applyh_on(ctx, vin, vout, nb, prec, flags, (cudaStream_t)stream);
}

// runs on the context's own stream and returns when the result is in vout
// (host pointers) or when the kernel has been queued (device pointers)
int bsg_applyh(bsg_ctx *ctx, const void *vin, void *vout, int nb, int prec, int flags) {
    if (!ctx) return BSG_ERR_ARG;
    return applyh_on(ctx, vin, vout, nb, prec, flags, ctx->stream);
}

int bsg_get_stats(const bsg_ctx *ctx, bsg_stats *st) {
    if (!ctx || !st) return BSG_ERR_ARG;
    *st = ctx->stats;
    return BSG_OK;
}

}  // extern "C"
