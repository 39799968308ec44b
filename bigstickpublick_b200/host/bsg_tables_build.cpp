// Host-side table builder: fills the BIGSTICK module arrays that bsg_create()
// consumes, for full (untruncated) M-scheme spaces.  CPU only; it plays the
// role of the Fortran host's setup (src/bigstick_main.f90:305-676), so that
// this project can produce the same kind of tables without a Fortran
// compiler.  See include/bsg_host.h for the list of reference stages.
//
// Conventions follow the reference:
//  * s.p. states are sorted by W, parity, |m| with the reference's selection
//    sort (src/bspstates.f90:110-225) and split into "left" (m<0, label -i)
//    and "right" (m>=0, label +i) halves (make_hspsqn, :235-332);
//  * an SD is a (left haiku, right haiku) pair; sectors are ordered by parity
//    then jz (ascending for protons, descending for neutrons,
//    src/bbasislib.f90:227-324); inside a sector SDs come in (right block,
//    left block) pairs with the left haiku as the slow index
//    (src/bjumplib_weld.f90:377-382); inside a block the haikus are in
//    count_create_haikus order (src/bbasis_haikus.f90:327-411, one W
//    section);
//  * basis index = pstart(ip) + nstart(in) (combinebasis,
//    src/bbasislib.f90:540-677);
//  * jump isd/fsd hold pstart/nstart values (bjumplib_weld.f90:791-792);
//    two-body jumps inside one sector keep only isd >= fsd (:414-420) and the
//    diagonal pair matrix element carries a factor 1/2 (btbme.f90:1402-1407);
//  * pairs are generated as count_create_pairs / count_create_pnpairs make
//    them and put in (M,par) sections, M descending, by sortpair's heap sorts
//    (src/btbme.f90:208-423, :548-703);
//  * uncoupled pp/nn matrix elements are packed lower triangles per (M,par)
//    section of pairs (bjumplib_weld.f90:635-642); pn ones are full squares
//    per (M,par) section, addressed by cpnpair(b,a)+dpnpair(d,c)
//    (btbmepn.f90:417-487);
//  * when there are at least two valence particles the single-particle
//    energies are folded into the two-body part with the factor 1/(A-1)
//    (src/bsppot.f90:20-238).
//
// The order of the jumps inside one sector jump is the builder's own (initial
// SDs in basis order); the reference's comes from its hop and chain lists
// (src/bjumplib_chains.f90, src/bhopslib.f90).  The GPU path never depends on
// that order.

#include "bsg_host.h"
#include "../csrc/ref_order.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <thread>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

namespace {

thread_local std::string g_err;
// host threads one build may use: set from the basis size once it is known
// (small systems build in one thread, so many builds can run side by side
// without oversubscribing the cores)
thread_local unsigned g_max_threads = 1;

// fn(i) for every i in [0, n) on up to g_max_threads host threads, indices
// taken from a shared counter; each index writes only what it owns, so the
// tables do not depend on the schedule
template <typename F>
void parallel_for(int64_t n, F fn) {
    const unsigned hw = std::max(1u, std::min(g_max_threads, std::thread::hardware_concurrency()));
    const int nt = (int)std::min<int64_t>((int64_t)hw, n);
    if (nt <= 1) {
        for (int64_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<int64_t> next{0};
    std::atomic<bool> oom{false};
    auto work = [&]() {
        try {
            for (int64_t i; (i = next.fetch_add(1)) < n && !oom;) fn(i);
        } catch (const std::bad_alloc &) {
            oom = true;
        }
    };
    std::vector<std::thread> th;
    for (int k = 1; k < nt; ++k) th.emplace_back(work);
    work();
    for (auto &x : th) x.join();
    if (oom) throw std::bad_alloc();
}

struct SPS {
    int nr, l, j2, m2, w, par, orb;
};

// ---------------------------------------------------------------- CG -------
// log n! for n < 256, filled when the library loads and read-only after, so
// several threads may build tables at the same time
struct LogFact {
    double v[256];
    LogFact() {
        v[0] = 0.0;
        for (int i = 1; i < 256; ++i) v[i] = v[i - 1] + std::log((double)i);
    }
};
const LogFact g_lfact_table;
const double *const g_lfact = g_lfact_table.v;
void init_lfact() {}
// <j1/2 m1/2 j2/2 m2/2 | J/2 M/2>, all arguments doubled (Racah's formula).
double cg2(int j1, int m1, int j2, int m2, int J, int M) {
    if (m1 + m2 != M) return 0.0;
    if (std::abs(m1) > j1 || std::abs(m2) > j2 || std::abs(M) > J) return 0.0;
    if (J > j1 + j2 || J < std::abs(j1 - j2)) return 0.0;
    if (((j1 + m1) & 1) || ((j2 + m2) & 1) || ((J + M) & 1) || ((j1 + j2 + J) & 1)) return 0.0;
    const int a = (j1 + j2 - J) / 2, b = (j1 - j2 + J) / 2, c = (-j1 + j2 + J) / 2;
    const int d = (j1 + j2 + J) / 2 + 1;
    double pre = 0.5 * (std::log((double)(J + 1)) + g_lfact[a] + g_lfact[b] + g_lfact[c] - g_lfact[d]);
    pre += 0.5 * (g_lfact[(j1 + m1) / 2] + g_lfact[(j1 - m1) / 2] + g_lfact[(j2 + m2) / 2] +
                  g_lfact[(j2 - m2) / 2] + g_lfact[(J + M) / 2] + g_lfact[(J - M) / 2]);
    double sum = 0.0;
    for (int k = 0; k <= 200; ++k) {
        const int t1 = a - k, t2 = (j1 - m1) / 2 - k, t3 = (j2 + m2) / 2 - k;
        const int t4 = (J - j2 + m1) / 2 + k, t5 = (J - j1 - m2) / 2 + k;
        if (t1 < 0 || t2 < 0 || t3 < 0) break;
        if (t4 < 0 || t5 < 0) continue;
        const double den = g_lfact[k] + g_lfact[t1] + g_lfact[t2] + g_lfact[t3] + g_lfact[t4] + g_lfact[t5];
        const double term = std::exp(pre - den);
        sum += (k & 1) ? -term : term;
    }
    return sum;
}

inline int popc(uint64_t x) { return __builtin_popcountll(x); }
// number of occupied states strictly below q
inline int nbelow(uint64_t bits, int q) { return popc(bits & ((q == 0) ? 0ull : ((1ull << q) - 1ull))); }

// ------------------------------------------------------- species basis -----
struct Haiku {
    uint64_t bits;  // over the half space (left: bit i = left state i)
    int jz2, par;
};
struct HBlock {
    int nh, pidx, jz2;
    std::vector<uint64_t> haikus;
};
struct Sector {
    int pidx, jz2;
    int64_t xsdstart = 0, xsdend = -1;  // 1-based
    std::vector<std::pair<int, int>> blocks;  // (right block, left block)
};
struct SpeciesBasis {
    int N = 0;
    int nl = 0, nr = 0;
    std::vector<SPS> left, right;       // hspsqn(-it,:), hspsqn(it,:)
    std::vector<int> q_orb, q_m2, q_par;  // per combined label q
    std::vector<HBlock> rblocks, lblocks;
    std::vector<Sector> sectors;
    std::vector<uint64_t> sd_bits;     // per SD (0-based index = isd-1)
    std::vector<int> sd_sector;        // 0-based sector of each SD
    std::unordered_map<uint64_t, int64_t> sd_index;  // bits -> 0-based SD index
    // the same map as a direct table over all occupation patterns when the
    // species has at most kDenseSps s.p. states (-1: not an SD of the basis);
    // the jump generators look up every candidate final SD
    std::vector<int64_t> sd_dense;
    int64_t find_sd(uint64_t bits) const {
        if (!sd_dense.empty()) return bits < sd_dense.size() ? sd_dense[bits] : -1;
        auto f = sd_index.find(bits);
        return f == sd_index.end() ? -1 : f->second;
    }
};

constexpr int kDenseSps = 22;   // 2^22 entries of 8 bytes at most per species

inline int pidx_of(int par) { return par > 0 ? 1 : 2; }
inline int par_of_idx(int p) { return p == 1 ? 1 : -1; }
inline int parmult(int p1, int p2) { return (p1 == p2) ? 1 : 2; }

// s.p. states: extract_sps + sort_spsqn + make_hspsqn
void make_sps(const bsg_model_spec *s, bool allsamepar, bool allsameW, SpeciesBasis &sb) {
    std::vector<SPS> sp;
    for (int i = 0; i < s->norb; ++i) {
        const bsg_orbit &o = s->orbits[i];
        for (int m = -o.j2; m <= o.j2; m += 2) {
            SPS x;
            x.nr = o.nr; x.l = o.l; x.j2 = o.j2; x.m2 = m; x.w = o.w;
            x.par = allsamepar ? 1 : ((o.l & 1) ? -1 : 1);
            x.orb = i;
            sp.push_back(x);
        }
    }
    const int n = (int)sp.size();
    // selection sort with swap on W (src/bspstates.f90:125-145)
    if (!allsameW) {
        for (int is = 0; is < n; ++is) {
            int k = is, w = sp[is].w;
            SPS tmp = sp[is];
            for (int j = is + 1; j < n; ++j)
                if (sp[j].w < w) { k = j; w = sp[j].w; tmp = sp[j]; }
            if (k != is) { sp[k] = sp[is]; sp[is] = tmp; }
        }
    }
    // on parity within each W (:149-181)
    if (!allsamepar) {
        int istart = 0;
        while (istart < n) {
            int iend = istart;
            for (int is = istart; is < n; ++is)
                if (sp[is].w == sp[istart].w) iend = is;
            for (int is = istart; is <= iend; ++is) {
                int k = is, par = sp[is].par;
                SPS tmp = sp[is];
                for (int j = is + 1; j <= iend; ++j)
                    if (sp[j].par < par) { k = j; par = sp[j].par; tmp = sp[j]; }
                if (k != is) { sp[k] = sp[is]; sp[is] = tmp; }
            }
            istart = iend + 1;
        }
    }
    // on |m| within each (W, par) (:185-213)
    {
        int istart = 0;
        while (istart < n) {
            int iend = istart;
            for (int is = istart; is < n; ++is)
                if (sp[is].w == sp[istart].w && sp[is].par == sp[istart].par) iend = is;
            for (int is = istart; is <= iend; ++is) {
                int k = is, m = sp[is].m2;
                SPS tmp = sp[is];
                for (int j = is + 1; j <= iend; ++j)
                    if (std::abs(sp[j].m2) < std::abs(m)) { k = j; m = sp[j].m2; tmp = sp[j]; }
                if (k != is) { sp[k] = sp[is]; sp[is] = tmp; }
            }
            istart = iend + 1;
        }
    }
    // split (make_hspsqn :254-271)
    sb.left.clear(); sb.right.clear();
    for (auto &x : sp) (x.m2 >= 0 ? sb.right : sb.left).push_back(x);
    sb.nl = (int)sb.left.size();
    sb.nr = (int)sb.right.size();
    sb.q_orb.resize(sb.nl + sb.nr);
    sb.q_m2.resize(sb.nl + sb.nr);
    sb.q_par.resize(sb.nl + sb.nr);
    for (int i = 0; i < sb.nl; ++i) { sb.q_orb[i] = sb.left[i].orb; sb.q_m2[i] = sb.left[i].m2; sb.q_par[i] = sb.left[i].par; }
    for (int i = 0; i < sb.nr; ++i) {
        sb.q_orb[sb.nl + i] = sb.right[i].orb; sb.q_m2[sb.nl + i] = sb.right[i].m2; sb.q_par[sb.nl + i] = sb.right[i].par;
    }
}

// all haikus of size k over `states`, grouped into blocks keyed (k, pidx, jz2),
// each block in the order count_create_haikus makes them
void make_blocks(const std::vector<SPS> &states, int kmin, int kmax, std::vector<HBlock> &blocks) {
    const int ns = (int)states.size();
    std::map<std::tuple<int, int, int>, std::vector<uint64_t>> groups;
    if (ns > 62) return;
    for (int k = kmin; k <= kmax; ++k) {
        if (k < 0 || k > ns) continue;
        // enumerate k-subsets in increasing bitmask order (Gosper's hack)
        if (k == 0) {
            groups[std::make_tuple(0, 1, 0)].push_back(0ull);
            continue;
        }
        uint64_t x = (1ull << k) - 1ull;
        const uint64_t lim = 1ull << ns;
        while (x < lim) {
            int jz = 0, par = 1;
            for (int i = 0; i < ns; ++i)
                if (x >> i & 1ull) { jz += states[i].m2; par *= states[i].par; }
            groups[std::make_tuple(k, pidx_of(par), jz)].push_back(x);
            const uint64_t c = x & (~x + 1ull), r = x + c;
            x = (((r ^ x) >> 2) / c) | r;
        }
    }
    blocks.clear();
    for (auto &g : groups) {  // std::map order: nh, parity index, jz ascending
        HBlock b;
        b.nh = std::get<0>(g.first);
        b.pidx = std::get<1>(g.first);
        b.jz2 = std::get<2>(g.first);
        b.haikus = std::move(g.second);
        // the reference's creation order inside the block
        std::sort(b.haikus.begin(), b.haikus.end(), [ns](uint64_t x, uint64_t y) {
            return bsg_order::haiku_rank(x, ns) < bsg_order::haiku_rank(y, ns);
        });
        blocks.push_back(std::move(b));
    }
}

int find_block(const std::vector<HBlock> &bl, int nh, int pidx, int jz2) {
    for (size_t i = 0; i < bl.size(); ++i)
        if (bl[i].nh == nh && bl[i].pidx == pidx && bl[i].jz2 == jz2) return (int)i;
    return -1;
}

// sector candidates (pidx, jz2) that some (right block, left block) pair reaches
std::map<std::pair<int, int>, int> sector_candidates(const SpeciesBasis &sb) {
    std::map<std::pair<int, int>, int> cand;
    for (auto &rb : sb.rblocks)
        for (auto &lb : sb.lblocks)
            if (rb.nh + lb.nh == sb.N) cand[{parmult(rb.pidx, lb.pidx), rb.jz2 + lb.jz2}] = 1;
    return cand;
}

// fill one sector's blocks and SD list (count_fill_sectors_w_blocks)
void fill_sector(SpeciesBasis &sb, Sector &sec, int64_t &next_sd) {
    sec.xsdstart = next_sd + 1;
    int nhmin = 1 << 30, nhmax = -1;
    for (auto &rb : sb.rblocks) { nhmin = std::min(nhmin, rb.nh); nhmax = std::max(nhmax, rb.nh); }
    for (int nh = nhmin; nh <= nhmax; ++nh) {
        const int nhc = sb.N - nh;
        for (int parh = 1; parh <= 2; ++parh) {
            const int parhc = parmult(sec.pidx, parh);
            std::vector<int> rbs;
            for (size_t i = 0; i < sb.rblocks.size(); ++i)
                if (sb.rblocks[i].nh == nh && sb.rblocks[i].pidx == parh) rbs.push_back((int)i);
            std::sort(rbs.begin(), rbs.end(), [&](int a, int b) { return sb.rblocks[a].jz2 < sb.rblocks[b].jz2; });
            for (int ir : rbs) {
                const int jzhc = sec.jz2 - sb.rblocks[ir].jz2;
                const int il = find_block(sb.lblocks, nhc, parhc, jzhc);
                if (il < 0) continue;
                sec.blocks.push_back({ir, il});
                const HBlock &R = sb.rblocks[ir], &L = sb.lblocks[il];
                for (uint64_t lh : L.haikus)       // left haiku: slow index
                    for (uint64_t rh : R.haikus) { // right haiku: fast index
                        const uint64_t bits = lh | (rh << sb.nl);
                        sb.sd_index[bits] = next_sd;
                        sb.sd_bits.push_back(bits);
                        sb.sd_sector.push_back(-1);
                        ++next_sd;
                    }
            }
        }
    }
    sec.xsdend = next_sd;
}

// ------------------------------------------------------------ jumps --------
struct SectJump {
    int is, fs;        // 0-based sectors
    int64_t nstart;    // 0-based offset into the jump arrays
    int64_t njumps;
    bool diag;
};
struct Jumps1 {
    std::vector<int64_t> isd, fsd;
    std::vector<int16_t> cop, dop;
    std::vector<int8_t> phase;
};
struct Jumps2 {
    std::vector<int64_t> isd, fsd;
    std::vector<int32_t> op;
    std::vector<int8_t> phase;
};
// two-body jumps of a three-body run: created / destroyed pair labels
// (src/bjumplib_weld.f90:771-775)
struct Jumps2P {
    std::vector<int64_t> isd, fsd;
    std::vector<int32_t> cop, dop;
    std::vector<int8_t> phase;
};

inline int signed_label(const SpeciesBasis &sb, int q) { return q < sb.nl ? -(q + 1) : (q - sb.nl + 1); }

// a^+_i a_k |s>, phase relative to the canonical ascending-label product
inline int phase1(uint64_t bits, int i, int k) {
    if (i == k) return 1;
    int p = nbelow(bits, k);
    const uint64_t b1 = bits & ~(1ull << k);
    p += nbelow(b1, i);
    return (p & 1) ? -1 : 1;
}
// a^+_i a^+_j a_l a_k |s> with i<j, k<l
inline int phase2(uint64_t bits, int i, int j, int k, int l) {
    int p = nbelow(bits, k);
    uint64_t b = bits & ~(1ull << k);
    p += nbelow(b, l);
    b &= ~(1ull << l);
    p += nbelow(b, j);
    b |= (1ull << j);
    p += nbelow(b, i);
    return (p & 1) ? -1 : 1;
}

// a^+_i a^+_j a^+_k a_n a_m a_l |s> with i<j<k, l<m<n
inline int phase3(uint64_t bits, int i, int j, int k, int l, int m, int n) {
    int p = nbelow(bits, l);
    uint64_t b = bits & ~(1ull << l);
    p += nbelow(b, m);
    b &= ~(1ull << m);
    p += nbelow(b, n);
    b &= ~(1ull << n);
    p += nbelow(b, k);
    b |= (1ull << k);
    p += nbelow(b, j);
    b |= (1ull << j);
    p += nbelow(b, i);
    return (p & 1) ? -1 : 1;
}

// ----------------------------------------------------- interaction ---------
struct Coupled {
    int norb = 0;
    std::vector<int> j2;
    std::map<std::tuple<int, int, int, int, int, int>, double> v;  // canonical key
    // canonical form and sign of V_JT(a,b,c,d)
    std::tuple<int, int, int, int, int, int> canon(int a, int b, int c, int d, int J, int T, int &sign) const {
        sign = 1;
        if (a < b) { std::swap(a, b); if ((((j2[a] + j2[b]) / 2 + J + T) & 1)) sign = -sign; }
        if (c < d) { std::swap(c, d); if ((((j2[c] + j2[d]) / 2 + J + T) & 1)) sign = -sign; }
        if (std::make_pair(a, b) < std::make_pair(c, d)) { std::swap(a, c); std::swap(b, d); }
        return std::make_tuple(a, b, c, d, J, T);
    }
    bool pair_ok(int a, int b, int J, int T) const {
        if (J > (j2[a] + j2[b]) / 2 || J < std::abs(j2[a] - j2[b]) / 2) return false;
        if (a == b && ((J + T) % 2 == 0)) return false;
        return true;
    }
    double get(int a, int b, int c, int d, int J, int T) const {
        if (!pair_ok(a, b, J, T) || !pair_ok(c, d, J, T)) return 0.0;
        int sg;
        auto key = canon(a, b, c, d, J, T, sg);
        auto it = v.find(key);
        if (it == v.end()) return 0.0;
        return sg * it->second;
    }
};

struct Pairs {
    // XX: pairs (q1<q2) ; PN: (qp, qn)
    std::vector<std::pair<int, int>> list;     // sorted order
    std::vector<int> M, pidx;                  // per sorted pair
    std::vector<int64_t> sec_first, sec_n, sec_mestart;  // per section
    std::vector<int> pair_sec;                 // section of each sorted pair
    std::map<std::pair<int, int>, int64_t> index;  // (q1,q2) -> 1-based sorted index
    std::vector<int64_t> dense;                    // same, dense [q1*ns2 + q2]
    int ns2 = 0;
    int64_t nmat = 0;
    void make_dense(int n1, int n2) {
        ns2 = n2;
        dense.assign((size_t)n1 * n2, 0);
        for (auto &kv : index) dense[(size_t)kv.first.first * n2 + kv.first.second] = kv.second;
    }
    int64_t at(int q1, int q2) const { return dense[(size_t)q1 * ns2 + q2]; }
};

// pairs q1 < q2 of one species in count_create_pairs order (the higher
// state outer, src/btbme.f90:208-308), then sortpair: sections of (M, parity)
// with M descending, in the order find_pair_start lays out the matrix
// elements (:726-785)
void make_xx_pairs(const SpeciesBasis &sb, Pairs &P) {
    const int ns = sb.nl + sb.nr;
    struct Tmp { int q1, q2, M, pidx; };
    std::vector<Tmp> v;
    for (int q2 = 1; q2 < ns; ++q2)
        for (int q1 = 0; q1 < q2; ++q1) {
            Tmp t;
            t.q1 = q1; t.q2 = q2;
            t.M = (sb.q_m2[q1] + sb.q_m2[q2]) / 2;
            t.pidx = pidx_of(sb.q_par[q1] * sb.q_par[q2]);
            v.push_back(t);
        }
    bsg_order::sortpair(v);
    P.list.clear(); P.M.clear(); P.pidx.clear(); P.pair_sec.clear();
    P.sec_first.clear(); P.sec_n.clear(); P.sec_mestart.clear(); P.index.clear();
    int64_t nme = 0;
    for (size_t i = 0; i < v.size(); ++i) {
        if (i == 0 || v[i].M != v[i - 1].M || v[i].pidx != v[i - 1].pidx) {
            if (!P.sec_n.empty()) nme += P.sec_n.back() * (P.sec_n.back() + 1) / 2;
            P.sec_first.push_back((int64_t)i + 1);  // 1-based first index
            P.sec_n.push_back(0);
            P.sec_mestart.push_back(nme);
        }
        P.sec_n.back() += 1;
        P.list.push_back({v[i].q1, v[i].q2});
        P.M.push_back(v[i].M);
        P.pidx.push_back(v[i].pidx);
        P.pair_sec.push_back((int)P.sec_n.size() - 1);
        P.index[{v[i].q1, v[i].q2}] = (int64_t)i + 1;
    }
    if (!P.sec_n.empty()) nme += P.sec_n.back() * (P.sec_n.back() + 1) / 2;
    P.nmat = nme;
    P.make_dense(ns, ns);
}

// itbme for sorted pair indices c, d (1-based, same section): triangle packing
inline int64_t xx_label(const Pairs &P, int64_t c, int64_t d) {
    const int s = P.pair_sec[c - 1];
    const int64_t iref = P.sec_first[s] - 1, istart = P.sec_mestart[s];
    const int64_t hi = std::max(c, d), lo = std::min(c, d);
    return istart + (hi - iref) * (hi - iref - 1) / 2 + lo - iref;
}

// (proton state, neutron state) pairs in count_create_pnpairs order (proton
// outer, src/btbme.f90:324-423), then sortpair as for like-particle pairs
// (src/btbmepn.f90:86); count_uncouplepn lays the squares out in that order
void make_pn_pairs(const SpeciesBasis &pb, const SpeciesBasis &nb, Pairs &P) {
    struct Tmp { int qp, qn, M, pidx; };
    std::vector<Tmp> v;
    const int nsp = pb.nl + pb.nr, nsn = nb.nl + nb.nr;
    for (int qp = 0; qp < nsp; ++qp)
        for (int qn = 0; qn < nsn; ++qn) {
            Tmp t;
            t.qp = qp; t.qn = qn;
            t.M = (pb.q_m2[qp] + nb.q_m2[qn]) / 2;
            t.pidx = pidx_of(pb.q_par[qp] * nb.q_par[qn]);
            v.push_back(t);
        }
    bsg_order::sortpair(v);
    P.list.clear(); P.M.clear(); P.pidx.clear(); P.pair_sec.clear();
    P.sec_first.clear(); P.sec_n.clear(); P.sec_mestart.clear(); P.index.clear();
    int64_t nme = 0;
    for (size_t i = 0; i < v.size(); ++i) {
        if (i == 0 || v[i].M != v[i - 1].M || v[i].pidx != v[i - 1].pidx) {
            if (!P.sec_n.empty()) nme += P.sec_n.back() * P.sec_n.back();
            P.sec_first.push_back((int64_t)i + 1);
            P.sec_n.push_back(0);
            P.sec_mestart.push_back(nme);
        }
        P.sec_n.back() += 1;
        P.list.push_back({v[i].qp, v[i].qn});
        P.M.push_back(v[i].M);
        P.pidx.push_back(v[i].pidx);
        P.pair_sec.push_back((int)P.sec_n.size() - 1);
        P.index[{v[i].qp, v[i].qn}] = (int64_t)i + 1;
    }
    if (!P.sec_n.empty()) nme += P.sec_n.back() * P.sec_n.back();
    P.nmat = nme;
    P.make_dense(nsp, nsn);
}

// --------------------------------------------------------- triplets --------
// Three-particle states of one kind in (M, parity) sections, as the
// reference's XXX3 / XXY lists (src/b3bmelib2.f90:430-560):
//  XXX: s.p. states q1<q2<q3 of one species, ordered by M, parity, then the
//       colex index C(q3,3)+C(q2,2)+q1 -- the index weld3b forms before
//       mapPPP / mapNNN (src/bjumplib_weld.f90:1108-1126); triangle-packed
//       labels per section as the pairs (:1149-1155);
//  XXY: a pair of species X (1-based pair label) and a s.p. state of
//       species Y, ordered by M, parity, pair, s.p. state; square sections
//       addressed by cXXYtriplet(pair, y) = start + (pos-1)*n and
//       dXXYtriplet = pos (assign_XXY_maps, src/b3bmelib2.f90:500-545).
struct Trips {
    std::vector<std::array<int, 3>> list;   // XXX: q1, q2, q3 ; XXY: pair, qy, 0
    std::vector<int> sec;                   // section of each sorted triplet
    std::vector<int64_t> sec_first, sec_n, sec_mestart;  // first: 1-based
    std::vector<int32_t> dense;             // XXX: colex -> 1-based sorted; XXY: (pair-1)*nsy + qy -> 1-based
    std::vector<std::vector<int32_t>> by_sec;  // sorted indices (1-based) per section
    int nsy = 0;
    int64_t nmat = 0;
};
inline int64_t colex3(int a, int b, int c) {  // a < b < c, 0-based
    return (int64_t)c * (c - 1) * (c - 2) / 6 + (int64_t)b * (b - 1) / 2 + a;
}
template <typename Tmp>
void sections_of(std::vector<Tmp> &v, Trips &T, bool square) {
    T.list.clear(); T.sec.clear(); T.sec_first.clear(); T.sec_n.clear(); T.sec_mestart.clear(); T.by_sec.clear();
    int64_t nme = 0;
    auto close = [&]() {
        if (T.sec_n.empty()) return;
        const int64_t n = T.sec_n.back();
        nme += square ? n * n : n * (n + 1) / 2;
    };
    for (size_t i = 0; i < v.size(); ++i) {
        if (i == 0 || v[i].m2 != v[i - 1].m2 || v[i].pidx != v[i - 1].pidx) {
            close();
            T.sec_first.push_back((int64_t)i + 1);
            T.sec_n.push_back(0);
            T.sec_mestart.push_back(nme);
            T.by_sec.emplace_back();
        }
        T.sec_n.back() += 1;
        T.list.push_back(v[i].key);
        T.sec.push_back((int)T.sec_n.size() - 1);
        T.by_sec.back().push_back((int32_t)i + 1);
    }
    close();
    T.nmat = nme;
}
void make_xxx(const SpeciesBasis &sb, Trips &T) {
    const int ns = sb.nl + sb.nr;
    struct Tmp { std::array<int, 3> key; int m2, pidx; int64_t cx; };
    std::vector<Tmp> v;
    for (int c = 2; c < ns; ++c)
        for (int b = 1; b < c; ++b)
            for (int a = 0; a < b; ++a)
                v.push_back({{a, b, c}, sb.q_m2[a] + sb.q_m2[b] + sb.q_m2[c],
                             pidx_of(sb.q_par[a] * sb.q_par[b] * sb.q_par[c]), colex3(a, b, c)});
    std::stable_sort(v.begin(), v.end(), [](const Tmp &x, const Tmp &y) {
        if (x.m2 != y.m2) return x.m2 < y.m2;
        if (x.pidx != y.pidx) return x.pidx < y.pidx;
        return x.cx < y.cx;
    });
    sections_of(v, T, false);
    T.dense.assign(ns >= 3 ? (size_t)colex3(ns - 3, ns - 2, ns - 1) + 1 : 0, 0);
    for (size_t i = 0; i < v.size(); ++i) T.dense[v[i].cx] = (int32_t)i + 1;
}
void make_xxy(const Pairs &PX, const SpeciesBasis &sy, Trips &T) {
    const int nsy = sy.nl + sy.nr;
    struct Tmp { std::array<int, 3> key; int m2, pidx; };
    std::vector<Tmp> v;
    for (size_t bb = 1; bb <= PX.list.size(); ++bb)
        for (int q = 0; q < nsy; ++q)
            v.push_back({{(int)bb, q, 0}, 2 * PX.M[bb - 1] + sy.q_m2[q],
                         pidx_of(par_of_idx(PX.pidx[bb - 1]) * sy.q_par[q])});
    std::stable_sort(v.begin(), v.end(), [](const Tmp &x, const Tmp &y) {
        if (x.m2 != y.m2) return x.m2 < y.m2;
        return x.pidx < y.pidx;
    });
    sections_of(v, T, true);
    T.nsy = nsy;
    T.dense.assign(PX.list.size() * (size_t)nsy, 0);
    for (size_t i = 0; i < v.size(); ++i) T.dense[(size_t)(v[i].key[0] - 1) * nsy + v[i].key[1]] = (int32_t)i + 1;
}
// label of sorted triplets c, d (1-based, same section) in a triangle section
inline int64_t xxx_label(const Trips &T, int64_t c, int64_t d) {
    const int s = T.sec[c - 1];
    const int64_t iref = T.sec_first[s] - 1, istart = T.sec_mestart[s];
    const int64_t hi = std::max(c, d), lo = std::min(c, d);
    return istart + (hi - iref) * (hi - iref - 1) / 2 + lo - iref;
}
// the seeded three-body part R(T, T') (bsg_host.h)
inline uint64_t mix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double r3(uint64_t seed, int kind, std::array<int, 3> k1, std::array<int, 3> k2) {
    if (k2 < k1) std::swap(k1, k2);
    uint64_t x = mix64(seed ^ (uint64_t)kind);
    for (int v : k1) x = mix64(x ^ (uint64_t)v);
    for (int v : k2) x = mix64(x ^ (uint64_t)v);
    return (double)(x >> 11) * 0x1.0p-52 - 1.0;
}

// ------------------------------------------------------------ sort ---------
// sort1bjumps / sort1bjumps_ins (src/bsortjumpslib.f90:190-290): shell sort
// with a fixed stride table, key = `key`, carried = the rest.
void shell_sort_1b(int64_t ndim, int64_t *other, int64_t *key, int16_t *cop, int16_t *dop, int8_t *ph) {
    static const int64_t strides[28] = {23422578909LL, 10410035071LL, 4626682254LL, 2056303224LL,
                                        913912544LL,  406183353LL,   180525935LL,  80233749LL,
                                        35659463LL,   15848650LL,    7043844LL,    3130597LL,
                                        1391376LL,    463792LL,      198768LL,     86961LL,
                                        33936LL,      13776LL,       4592LL,       1968LL,
                                        861LL,        336LL,         112LL,        48LL,
                                        21LL,         7LL,           3LL,          1LL};
    for (int ks = 0; ks < 28; ++ks) {
        const int64_t stride = strides[ks];
        if (stride > ndim) continue;
        for (int64_t off = 0; off < stride; ++off) {
            // Fortran: do j = off+stride+1, ndim, stride  (1-based)
            for (int64_t j = off + stride + 1; j <= ndim; j += stride) {
                const int64_t s_o = other[j - 1], s_k = key[j - 1];
                const int16_t s_c = cop[j - 1], s_d = dop[j - 1];
                const int8_t s_p = ph[j - 1];
                int64_t k = j, i = k - stride;
                while (i > 0) {
                    if (key[i - 1] <= s_k) break;
                    other[k - 1] = other[i - 1]; key[k - 1] = key[i - 1];
                    cop[k - 1] = cop[i - 1]; dop[k - 1] = dop[i - 1]; ph[k - 1] = ph[i - 1];
                    k = i;
                    i -= stride;
                }
                other[k - 1] = s_o; key[k - 1] = s_k; cop[k - 1] = s_c; dop[k - 1] = s_d; ph[k - 1] = s_p;
            }
        }
    }
}

// --------------------------------------------------------- container -------
struct Built {
    SpeciesBasis pb, nb;
    std::vector<int64_t> pstart, nstart;
    Jumps1 p1, n1;
    Jumps2 p2, n2;
    std::vector<SectJump> p1sj, n1sj, p2sj, n2sj;
    std::vector<float> hmatpp, hmatnn, hmatpn;
    std::vector<int64_t> cpn, dpn;
    std::vector<float> pspe_h, nspe_h;
    std::vector<int32_t> optype, hchar;
    std::vector<int64_t> pxstart, pxend, nxstart, nxend, cstride;
    std::vector<int64_t> ps_start, ps_end, ns_start, ns_end;
    std::vector<int32_t> ps_jz, ps_par, ns_jz, ns_par, ps_conj;
    std::vector<int32_t> spo_p, spm_p, spo_n, spm_n;
    Pairs ppairs, npairs, pnpairs;
    // one-body density jumps (Delta Jz = 0 sector jumps) and their bundles
    Jumps1 dp1, dn1;
    std::vector<int32_t> d_optype, d_hchar;
    std::vector<int64_t> d_pxstart, d_pxend, d_nxstart, d_nxend, d_cstride;
    // chain-rule bookkeeping: per matrix element, list of (tbme line, coef)
    std::vector<std::vector<std::pair<int, double>>> jac_pp, jac_nn, jac_pn;
    std::vector<std::vector<std::pair<int, double>>> jspe_pp, jspe_nn, jspe_pn;
    int ntbme = 0, norb = 0;
    // uncoupled two-body interaction in double, without the folded s.p.
    // energies and without the diagonal halving: vxx[0] pp, vxx[1] nn by
    // triangle label, vpn by square label
    std::vector<double> vxx[2], vpn;
    // three-body run (bsg_host_build3)
    bool three = false;
    Jumps2P p2x, n2x;                 // two-body jumps with pair labels (PPN protons, PNN neutrons)
    Jumps2 p3, n3;                    // three-body jumps inside a sector
    std::vector<float> hmatppp, hmatnnn, hmatppn, hmatpnn;
    std::vector<int32_t> cppn, dppn, cpnn, dpnn;
    bsg_tables3 t3{};
};

// coupled matrix element table with per-line provenance for the jacobian
struct Interaction {
    Coupled C;
    // canonical key -> list of (tbme line, sign) contributing to it
    std::map<std::tuple<int, int, int, int, int, int>, std::vector<std::pair<int, int>>> prov;
    // the same two maps as dense arrays over canonical (a, b, c, d, J, T):
    // the uncoupling asks for each element many times (once per m-scheme
    // pair-pair and J), so the lookups must not walk a tree
    int nj = 0;
    std::vector<double> dv;
    std::vector<uint8_t> dhas;
    std::vector<int32_t> dp0, dp1;                 // provenance range per entry
    std::vector<std::pair<int, int>> dprov;
    size_t slot(int a, int b, int c, int d, int J, int T) const {
        const size_t n = (size_t)C.norb;
        return (((((size_t)a * n + b) * n + c) * n + d) * (size_t)nj + J) * 2 + T;
    }
    void finalize() {
        int jmax = 0;
        for (int j : C.j2) jmax = std::max(jmax, j);
        nj = jmax + 1;
        const size_t n = (size_t)C.norb, tot = n * n * n * n * (size_t)nj * 2;
        dv.assign(tot, 0.0);
        dhas.assign(tot, 0);
        dp0.assign(tot, 0);
        dp1.assign(tot, 0);
        dprov.clear();
        for (auto &kv : C.v) {
            const auto &k = kv.first;
            const size_t q = slot(std::get<0>(k), std::get<1>(k), std::get<2>(k), std::get<3>(k), std::get<4>(k),
                                  std::get<5>(k));
            dv[q] = kv.second;
            dhas[q] = 1;
            dp0[q] = (int32_t)dprov.size();
            auto pit = prov.find(k);
            if (pit != prov.end()) dprov.insert(dprov.end(), pit->second.begin(), pit->second.end());
            dp1[q] = (int32_t)dprov.size();
        }
    }
};

// V_JT(a,b,c,d) as a linear combination of file lines: returns value, and
// appends (line, coef) scaled by `w`
double coupled_with_prov(const Interaction &I, int a, int b, int c, int d, int J, int T, double w,
                         std::vector<std::pair<int, double>> *acc) {
    const Coupled &C = I.C;
    if (!C.pair_ok(a, b, J, T) || !C.pair_ok(c, d, J, T)) return 0.0;
    int sg;
    const auto key = C.canon(a, b, c, d, J, T, sg);
    const size_t q = I.slot(std::get<0>(key), std::get<1>(key), std::get<2>(key), std::get<3>(key), J, T);
    if (!I.dhas[q]) return 0.0;
    if (acc)
        for (int32_t p = I.dp0[q]; p < I.dp1[q]; ++p) acc->push_back({I.dprov[p].first, w * sg * I.dprov[p].second});
    return sg * I.dv[q];
}

// sum the coefficients of each file line (in their order of appearance),
// ascending lines, zeros dropped
void compress(std::vector<std::pair<int, double>> &v) {
    std::stable_sort(v.begin(), v.end(),
                     [](const std::pair<int, double> &x, const std::pair<int, double> &y) { return x.first < y.first; });
    size_t out = 0;
    for (size_t i = 0; i < v.size();) {
        const int line = v[i].first;
        double sum = 0.0;
        for (; i < v.size() && v[i].first == line; ++i) sum += v[i].second;
        if (sum != 0.0) v[out++] = {line, sum};
    }
    v.resize(out);
}

int build(const bsg_model_spec *s, const bsg_model3_spec *s3, Built &B) {
    init_lfact();
    g_max_threads = 1;
    const bool three = (s3 != nullptr);
    B.three = three;
    if (!s || s->norb <= 0 || !s->orbits) { g_err = "bad model spec"; return BSG_ERR_ARG; }
    if (s->np < 0 || s->nn < 0) { g_err = "negative particle number"; return BSG_ERR_ARG; }
    B.norb = s->norb;
    B.ntbme = s->ntbme;
    bool allsamepar = true, allsameW = true;
    for (int i = 0; i < s->norb; ++i) {
        if ((s->orbits[i].l & 1) != (s->orbits[0].l & 1)) allsamepar = false;
        if (s->orbits[i].w != s->orbits[0].w) allsameW = false;
        if (s->orbits[i].j2 <= 0 || (s->orbits[i].j2 & 1) == 0) { g_err = "orbit j must be half-integer"; return BSG_ERR_ARG; }
    }
    const int iparity_idx = allsamepar ? 1 : pidx_of(s->parity >= 0 ? 1 : -1);

    // ---- s.p. states and haiku blocks per species
    SpeciesBasis *sbs[2] = {&B.pb, &B.nb};
    const int Ns[2] = {s->np, s->nn};
    for (int it = 0; it < 2; ++it) {
        SpeciesBasis &sb = *sbs[it];
        sb.N = Ns[it];
        make_sps(s, allsamepar, allsameW, sb);
        if (sb.nl + sb.nr > 62) { g_err = "more than 62 s.p. states per species"; return BSG_ERR_UNSUPPORTED; }
        if (sb.N > sb.nl + sb.nr) { g_err = "too many particles for the space"; return BSG_ERR_ARG; }
        make_blocks(sb.right, std::max(0, sb.N - sb.nl), std::min(sb.N, sb.nr), sb.rblocks);
        make_blocks(sb.left, std::max(0, sb.N - sb.nr), std::min(sb.N, sb.nl), sb.lblocks);
    }
    // ---- sectors: protons parity 1..2 / jz ascending; neutrons jz descending
    auto pc = sector_candidates(B.pb), nc = sector_candidates(B.nb);
    std::vector<std::pair<int, int>> psec, nsec;
    for (int p = 1; p <= 2; ++p) {
        std::vector<int> jzs;
        for (auto &c : pc)
            if (c.first.first == p) {
                const int jzn = s->jz2 - c.first.second;
                const int pn = parmult(iparity_idx, p);
                if (nc.count({pn, jzn})) jzs.push_back(c.first.second);
            }
        std::sort(jzs.begin(), jzs.end());
        for (int jz : jzs) psec.push_back({p, jz});
    }
    {
        std::vector<int> porder = (iparity_idx == 1) ? std::vector<int>{1, 2} : std::vector<int>{2, 1};
        for (int p : porder) {
            std::vector<int> jzs;
            for (auto &c : nc)
                if (c.first.first == p) {
                    const int jzp = s->jz2 - c.first.second;
                    const int pp = parmult(iparity_idx, p);
                    if (pc.count({pp, jzp})) jzs.push_back(c.first.second);
                }
            std::sort(jzs.begin(), jzs.end(), std::greater<int>());
            for (int jz : jzs) nsec.push_back({p, jz});
        }
    }
    if (psec.empty() || nsec.empty()) { g_err = "no basis states for this Jz/parity"; return BSG_ERR_ARG; }
    for (int it = 0; it < 2; ++it) {
        SpeciesBasis &sb = *sbs[it];
        auto &lst = it == 0 ? psec : nsec;
        int64_t next = 0;
        for (auto &ps : lst) {
            Sector sec;
            sec.pidx = ps.first;
            sec.jz2 = ps.second;
            fill_sector(sb, sec, next);
            for (int64_t k = sec.xsdstart - 1; k < sec.xsdend; ++k) sb.sd_sector[k] = (int)sb.sectors.size();
            sb.sectors.push_back(std::move(sec));
        }
    }
    const int nps = (int)B.pb.sectors.size(), nns = (int)B.nb.sectors.size();
    std::vector<int> pconj(nps, -1), nconj(nns, -1);
    for (int a = 0; a < nps; ++a)
        for (int b = 0; b < nns; ++b)
            if (B.pb.sectors[a].jz2 + B.nb.sectors[b].jz2 == s->jz2 &&
                parmult(B.pb.sectors[a].pidx, B.nb.sectors[b].pidx) == iparity_idx) {
                pconj[a] = b;
                nconj[b] = a;
            }
    for (int a = 0; a < nps; ++a)
        if (pconj[a] < 0) { g_err = "proton sector without conjugate"; return BSG_ERR_BAD_TABLE; }

    // ---- combinebasis (src/bbasislib.f90:540-677)
    const int64_t nsdp = (int64_t)B.pb.sd_bits.size(), nsdn = (int64_t)B.nb.sd_bits.size();
    B.pstart.assign(nsdp, -1);
    B.nstart.assign(nsdn, -1);
    int64_t dimbasis = 1, pcount = 0, ncount = 0;
    for (int is = 0; is < nps; ++is) {
        const Sector &ps = B.pb.sectors[is];
        const Sector &ns = B.nb.sectors[pconj[is]];
        const int64_t ndim = ns.xsdend - ns.xsdstart + 1;
        if (nconj[pconj[is]] == is) {
            for (int64_t in = 1; in <= ndim; ++in) B.nstart[ncount++] = in;
        }
        const int64_t pdim = ps.xsdend - ps.xsdstart + 1;
        for (int64_t ip = 0; ip < pdim; ++ip) {
            B.pstart[pcount++] = dimbasis - 1;
            dimbasis += ndim;
        }
    }
    dimbasis -= 1;
    if (pcount != nsdp || ncount != nsdn) { g_err = "combinebasis count mismatch"; return BSG_ERR_BAD_TABLE; }
    g_max_threads = dimbasis >= ((int64_t)1 << 18) ? 32u : 1u;

    // ---- interaction: coupled V_JT canonicalized with provenance
    Interaction I;
    I.C.norb = s->norb;
    for (int i = 0; i < s->norb; ++i) I.C.j2.push_back(s->orbits[i].j2);
    for (int i = 0; i < s->ntbme; ++i) {
        const bsg_tbme &t = s->tbme[i];
        const int a = t.a - 1, b = t.b - 1, c = t.c - 1, d = t.d - 1;
        if (a < 0 || b < 0 || c < 0 || d < 0 || a >= s->norb || b >= s->norb || c >= s->norb || d >= s->norb) {
            g_err = "TBME orbit label out of range";
            return BSG_ERR_ARG;
        }
        if (!I.C.pair_ok(a, b, t.J, t.T) || !I.C.pair_ok(c, d, t.J, t.T)) continue;
        int sg;
        auto key = I.C.canon(a, b, c, d, t.J, t.T, sg);
        I.C.v[key] += sg * t.v;
        I.prov[key].push_back({i, sg});
    }
    I.finalize();
    const double vscale = s->tbme_scale;
    const int A = s->np + s->nn;
    // a three-body run keeps the s.p. energies as SPE bundles
    const bool call_spe = (A <= 1) || three;
    if (three && A < 3) { g_err = "a three-body run needs at least three valence particles"; return BSG_ERR_ARG; }
    const double afac = (A > 1) ? 1.0 / (double)(A - 1) : 0.0;
    std::vector<double> spe(s->norb, 0.0);
    for (int i = 0; i < s->norb; ++i) spe[i] = s->spe ? s->spe_scale * s->spe[i] : 0.0;

    // ---- pp / nn uncoupled (uncoupleXXtbme, src/btbme.f90:1209-1551)
    const int nspsp = B.pb.nl + B.pb.nr;
    for (int it = 0; it < 2; ++it) {
        SpeciesBasis &sb = *sbs[it];
        Pairs &P = it == 0 ? B.ppairs : B.npairs;
        make_xx_pairs(sb, P);
        std::vector<float> &H = it == 0 ? B.hmatpp : B.hmatnn;
        auto &jac = it == 0 ? B.jac_pp : B.jac_nn;
        auto &jspe = it == 0 ? B.jspe_pp : B.jspe_nn;
        H.assign(P.nmat, 0.0f);
        jac.assign(P.nmat, {});
        jspe.assign(P.nmat, {});
        B.vxx[it].assign(P.nmat, 0.0);
        if (sb.N < 2 && !three) continue;
        for (size_t s_ = 0; s_ < P.sec_n.size(); ++s_) {
            const int64_t first = P.sec_first[s_], n = P.sec_n[s_];
            for (int64_t c = first; c < first + n; ++c)
                for (int64_t d = first; d <= c; ++d) {
                    const int64_t lab = xx_label(P, c, d);
                    const int i = P.list[c - 1].first, j = P.list[c - 1].second;
                    const int k = P.list[d - 1].first, l = P.list[d - 1].second;
                    const int a = sb.q_orb[i], b = sb.q_orb[j], cc = sb.q_orb[k], dd = sb.q_orb[l];
                    const int ja = I.C.j2[a], jb = I.C.j2[b], jc = I.C.j2[cc], jd = I.C.j2[dd];
                    const int M2 = sb.q_m2[i] + sb.q_m2[j];
                    const double zab = (a == b) ? std::sqrt(2.0) : 1.0, zcd = (cc == dd) ? std::sqrt(2.0) : 1.0;
                    double v = 0.0;
                    std::vector<std::pair<int, double>> pv;
                    for (int J = 0; J <= 20; ++J) {
                        const double cgab = cg2(ja, sb.q_m2[i], jb, sb.q_m2[j], 2 * J, M2);
                        if (cgab == 0.0) continue;
                        const double cgcd = cg2(jc, sb.q_m2[k], jd, sb.q_m2[l], 2 * J, M2);
                        if (cgcd == 0.0) continue;
                        const double w = zab * zcd * cgab * cgcd * vscale;
                        v += w * coupled_with_prov(I, a, b, cc, dd, J, 1, w, &pv);
                    }
                    B.vxx[it][lab - 1] = v;
                    std::vector<std::pair<int, double>> ps;
                    if (c == d) {  // SPE folded into the diagonal pair (bsppot.f90:83-106)
                        v += afac * (spe[a] + spe[b]);
                        ps.push_back({a, afac * s->spe_scale});
                        ps.push_back({b, afac * s->spe_scale});
                        v *= 0.5;  // hermitian doubling of diagonal jumps
                        for (auto &x : pv) x.second *= 0.5;
                        for (auto &x : ps) x.second *= 0.5;
                    }
                    H[lab - 1] = (float)v;
                    compress(pv);
                    compress(ps);
                    jac[lab - 1] = std::move(pv);
                    jspe[lab - 1] = std::move(ps);
                }
        }
    }
    // ---- pn uncoupled (count_uncouplepn, src/btbmepn.f90:177-587)
    make_pn_pairs(B.pb, B.nb, B.pnpairs);
    {
        Pairs &P = B.pnpairs;
        const int pl = B.pb.nl, pr = B.pb.nr, nl = B.nb.nl, nr = B.nb.nr;
        const int64_t ld = (int64_t)(nl + nr + 1);
        B.cpn.assign(ld * (pl + pr + 1), 0);
        B.dpn.assign(ld * (pl + pr + 1), 0);
        B.hmatpn.assign(P.nmat, 0.0f);
        B.jac_pn.assign(P.nmat, {});
        B.jspe_pn.assign(P.nmat, {});
        B.vpn.assign(P.nmat, 0.0);
        const bool have_pn = (s->np >= 1 && s->nn >= 1) || three;
        for (size_t s_ = 0; s_ < P.sec_n.size(); ++s_) {
            const int64_t first = P.sec_first[s_], n = P.sec_n[s_], nme = P.sec_mestart[s_];
            for (int64_t pos = 1; pos <= n; ++pos) {
                const int qp = P.list[first + pos - 2].first, qn = P.list[first + pos - 2].second;
                const int sp = signed_label(B.pb, qp), sn = signed_label(B.nb, qn);
                const int64_t idx = (int64_t)(sn + nl) + (int64_t)(sp + pl) * ld;
                B.cpn[idx] = (pos - 1) * n;
                B.dpn[idx] = pos + nme;
            }
            if (!have_pn) continue;
            // (ja ma, jb mb | J M) of every pair of the section, J = 0..20:
            // each appears in n matrix elements as the bra and n as the ket
            constexpr int kJ = 21;
            std::vector<double> cgt((size_t)n * kJ);
            for (int64_t pos = 1; pos <= n; ++pos) {
                const int qp = P.list[first + pos - 2].first, qn = P.list[first + pos - 2].second;
                const int jp = I.C.j2[B.pb.q_orb[qp]], jn = I.C.j2[B.nb.q_orb[qn]];
                const int m2 = B.pb.q_m2[qp] + B.nb.q_m2[qn];
                for (int J = 0; J < kJ; ++J)
                    cgt[(size_t)(pos - 1) * kJ + J] = cg2(jp, B.pb.q_m2[qp], jn, B.nb.q_m2[qn], 2 * J, m2);
            }
            for (int64_t cpos = 1; cpos <= n; ++cpos)
                for (int64_t dpos = 1; dpos <= n; ++dpos) {
                    const int64_t lab = nme + (cpos - 1) * n + dpos;
                    const int qa = P.list[first + cpos - 2].first, qb = P.list[first + cpos - 2].second;
                    const int qc = P.list[first + dpos - 2].first, qd = P.list[first + dpos - 2].second;
                    const int a = B.pb.q_orb[qa], b = B.nb.q_orb[qb], c = B.pb.q_orb[qc], d = B.nb.q_orb[qd];
                    const double zab = (a == b) ? std::sqrt(2.0) : 1.0, zcd = (c == d) ? std::sqrt(2.0) : 1.0;
                    double v = 0.0;
                    std::vector<std::pair<int, double>> pv;
                    for (int J = 0; J < kJ; ++J) {
                        const double cgab = cgt[(size_t)(cpos - 1) * kJ + J];
                        if (cgab == 0.0) continue;
                        const double cgcd = cgt[(size_t)(dpos - 1) * kJ + J];
                        if (cgcd == 0.0) continue;
                        const double w = 0.5 * zab * zcd * cgab * cgcd * vscale;
                        for (int T = 0; T <= 1; ++T) v += w * coupled_with_prov(I, a, b, c, d, J, T, w, &pv);
                    }
                    B.vpn[lab - 1] = v;
                    std::vector<std::pair<int, double>> ps;
                    if (cpos == dpos) {  // SPE folded into pn (bsppot.f90:185-226)
                        v += afac * (spe[a] + spe[b]);
                        ps.push_back({a, afac * s->spe_scale});
                        ps.push_back({b, afac * s->spe_scale});
                    }
                    B.hmatpn[lab - 1] = (float)v;
                    compress(pv);
                    compress(ps);
                    B.jac_pn[lab - 1] = std::move(pv);
                    B.jspe_pn[lab - 1] = std::move(ps);
                }
        }
    }
    (void)nspsp;

    // ---- jumps
    for (SpeciesBasis *sbp : sbs) {
        SpeciesBasis &sb = *sbp;
        const int ns = sb.nl + sb.nr;
        sb.sd_dense.clear();
        if (ns <= kDenseSps) {
            sb.sd_dense.assign((size_t)1 << ns, -1);
            for (size_t i = 0; i < sb.sd_bits.size(); ++i) sb.sd_dense[sb.sd_bits[i]] = (int64_t)i;
        }
    }
    // one-body: proton sector jumps (is >= fs), each with its conjugate
    // neutron sector jump (conj(is) -> conj(fs))
    // the one-body jumps out of a sector, generated in one pass over its SDs
    // (SD, then annihilated k, then created i) and bucketed by the final
    // sector; gen1 appends one bucket, so each (is, fs) keeps that order
    std::map<std::pair<const SpeciesBasis *, int>, std::vector<Jumps1>> jumps1_from;
    // every one-body jump out of sector `is`, bucketed by final sector
    auto jumps1_out = [&](const SpeciesBasis &sb, const std::vector<int64_t> &xstart, int is) {
        std::vector<Jumps1> by(sb.sectors.size());
        const Sector &S = sb.sectors[is];
        const int ns = sb.nl + sb.nr;
        for (int64_t sd = S.xsdstart - 1; sd < S.xsdend; ++sd) {
            const uint64_t bits = sb.sd_bits[sd];
            for (int k = 0; k < ns; ++k) {
                if (!(bits >> k & 1ull)) continue;
                for (int i = 0; i < ns; ++i) {
                    if (i != k && (bits >> i & 1ull)) continue;
                    const uint64_t nb2 = (bits & ~(1ull << k)) | (1ull << i);
                    const int64_t f = sb.find_sd(nb2);
                    if (f < 0) continue;
                    Jumps1 &B1 = by[sb.sd_sector[f]];
                    B1.isd.push_back(xstart[sd]);
                    B1.fsd.push_back(xstart[f]);
                    B1.cop.push_back((int16_t)signed_label(sb, i));
                    B1.dop.push_back((int16_t)signed_label(sb, k));
                    B1.phase.push_back((int8_t)phase1(bits, i, k));
                }
            }
        }
        return by;
    };
    // fill the cache for every source sector of both species on host threads
    // (the generators below then only copy buckets)
    if (s->np >= 1 || s->nn >= 1) {
        std::vector<std::pair<SpeciesBasis *, int>> srcs;
        for (int is = 0; is < nps; ++is) srcs.push_back({&B.pb, is});
        for (int is = 0; is < nns; ++is) srcs.push_back({&B.nb, is});
        std::vector<std::vector<Jumps1>> made(srcs.size());
        parallel_for((int64_t)srcs.size(), [&](int64_t j) {
            const SpeciesBasis &sb = *srcs[j].first;
            made[j] = jumps1_out(sb, &sb == &B.pb ? B.pstart : B.nstart, srcs[j].second);
        });
        for (size_t j = 0; j < srcs.size(); ++j)
            jumps1_from.emplace(std::make_pair((const SpeciesBasis *)srcs[j].first, srcs[j].second), std::move(made[j]));
    }
    auto gen1 = [&](SpeciesBasis &sb, const std::vector<int64_t> &xstart, int is, int fs, Jumps1 &J) {
        auto key = std::make_pair((const SpeciesBasis *)&sb, is);
        auto it = jumps1_from.find(key);
        if (it == jumps1_from.end()) it = jumps1_from.emplace(key, jumps1_out(sb, xstart, is)).first;
        const Jumps1 &src = it->second[fs];
        J.isd.insert(J.isd.end(), src.isd.begin(), src.isd.end());
        J.fsd.insert(J.fsd.end(), src.fsd.begin(), src.fsd.end());
        J.cop.insert(J.cop.end(), src.cop.begin(), src.cop.end());
        J.dop.insert(J.dop.end(), src.dop.begin(), src.dop.end());
        J.phase.insert(J.phase.end(), src.phase.begin(), src.phase.end());
        return (int64_t)src.isd.size();
    };
    // pairs (i < j) of each pair section (M, parity), in (i, j) order: the
    // creation pairs a two-body jump can use for a given annihilated pair
    auto pairs_by_section = [](const SpeciesBasis &sb, const Pairs &P) {
        const int ns = sb.nl + sb.nr;
        std::vector<std::vector<std::pair<int, int>>> by(P.sec_n.size());
        for (int i = 0; i < ns; ++i)
            for (int j = i + 1; j < ns; ++j) by[P.pair_sec[P.at(i, j) - 1]].push_back({i, j});
        return by;
    };
    auto gen2 = [&](SpeciesBasis &sb, const std::vector<int64_t> &xstart, const Pairs &P,
                    const std::vector<std::vector<std::pair<int, int>>> &by_sec, int is, int fs, Jumps2 &J) {
        int64_t cnt = 0;
        const Sector &S = sb.sectors[is];
        const int ns = sb.nl + sb.nr;
        const bool halve = (is == fs);
        std::vector<int> occ;
        for (int64_t sd = S.xsdstart - 1; sd < S.xsdend; ++sd) {
            const uint64_t bits = sb.sd_bits[sd];
            occ.clear();
            for (int q = 0; q < ns; ++q)
                if (bits >> q & 1ull) occ.push_back(q);
            for (size_t x = 0; x < occ.size(); ++x)
                for (size_t y = x + 1; y < occ.size(); ++y) {
                    const int k = occ[x], l = occ[y];
                    const uint64_t rest = bits & ~(1ull << k) & ~(1ull << l);
                    const int64_t dpair = P.at(k, l);
                    for (const auto &ij : by_sec[P.pair_sec[dpair - 1]]) {   // same M, parity
                        const int i = ij.first, j = ij.second;
                        if ((rest >> i & 1ull) || (rest >> j & 1ull)) continue;
                        const int64_t cpair = P.at(i, j);
                        const uint64_t nb2 = rest | (1ull << i) | (1ull << j);
                        const int64_t f = sb.find_sd(nb2);
                        if (f < 0 || sb.sd_sector[f] != fs) continue;
                        if (halve && sd < f) continue;  // keep isd >= fsd
                        J.isd.push_back(xstart[sd]);
                        J.fsd.push_back(xstart[f]);
                        J.op.push_back((int32_t)xx_label(P, cpair, dpair));
                        J.phase.push_back((int8_t)phase2(bits, i, j, k, l));
                        ++cnt;
                    }
                }
        }
        return cnt;
    };
    std::map<std::pair<int, int>, int> n1sj_of;
    for (int is = 0; is < nps; ++is)
        for (int fs = 0; fs <= is; ++fs) {
            if (s->np < 1 || s->nn < 1) continue;
            SectJump sj;
            sj.is = is; sj.fs = fs; sj.diag = (is == fs);
            sj.nstart = (int64_t)B.p1.isd.size();
            sj.njumps = gen1(B.pb, B.pstart, is, fs, B.p1);
            if (sj.njumps == 0) continue;
            const int in = pconj[is], fn = pconj[fs];
            if (!n1sj_of.count({in, fn})) {
                SectJump nj;
                nj.is = in; nj.fs = fn; nj.diag = (in == fn);
                nj.nstart = (int64_t)B.n1.isd.size();
                nj.njumps = gen1(B.nb, B.nstart, in, fn, B.n1);
                n1sj_of[{in, fn}] = (int)B.n1sj.size();
                B.n1sj.push_back(nj);
            }
            B.p1sj.push_back(sj);
        }
    // two-body jumps inside each sector: sectors on host threads, appended in
    // sector order
    auto two_body = [&](SpeciesBasis &sb, const std::vector<int64_t> &xstart, const Pairs &P, int nsec, Jumps2 &out,
                        std::vector<SectJump> &sjs) {
        const auto by_sec = pairs_by_section(sb, P);
        std::vector<Jumps2> per(nsec);
        parallel_for(nsec, [&](int64_t is) { gen2(sb, xstart, P, by_sec, (int)is, (int)is, per[is]); });
        for (int is = 0; is < nsec; ++is) {
            SectJump sj;
            sj.is = is; sj.fs = is; sj.diag = true;
            sj.nstart = (int64_t)out.isd.size();
            sj.njumps = (int64_t)per[is].isd.size();
            if (sj.njumps == 0) continue;
            out.isd.insert(out.isd.end(), per[is].isd.begin(), per[is].isd.end());
            out.fsd.insert(out.fsd.end(), per[is].fsd.begin(), per[is].fsd.end());
            out.op.insert(out.op.end(), per[is].op.begin(), per[is].op.end());
            out.phase.insert(out.phase.end(), per[is].phase.begin(), per[is].phase.end());
            sjs.push_back(sj);
        }
    };
    if (s->np >= 2 && !three) two_body(B.pb, B.pstart, B.ppairs, nps, B.p2, B.p2sj);
    if (s->nn >= 2 && !three) two_body(B.nb, B.nstart, B.npairs, nns, B.n2, B.n2sj);

    // ---- three-body run: triplet tables, matrix elements and jumps
    std::vector<SectJump> p3sj, n3sj, p2xsj, n2xsj;
    std::vector<int> p2x_n1;      // neutron one-body sector jump of each PPN sector jump
    std::vector<int> pnn_p1, pnn_n2x;  // PNN: proton one-body / neutron two-body sector jumps
    if (three) {
        Trips Tppp, Tnnn, Tppn, Tpnn;
        make_xxx(B.pb, Tppp);
        make_xxx(B.nb, Tnnn);
        make_xxy(B.ppairs, B.nb, Tppn);
        make_xxy(B.npairs, B.pb, Tpnn);
        const double w2 = s3->w2 / (double)(A - 2), w3 = s3->w3;
        const uint64_t seed = s3->seed;
        // uncoupled two-body interaction between pair labels / pn labels
        auto vxx = [&](int it, int64_t c, int64_t d) -> double {
            const Pairs &P = it == 0 ? B.ppairs : B.npairs;
            if (P.pair_sec[c - 1] != P.pair_sec[d - 1]) return 0.0;
            return B.vxx[it][xx_label(P, c, d) - 1];
        };
        auto vpn = [&](int qp, int qn, int qpp, int qnn) -> double {
            const Pairs &P = B.pnpairs;
            const int64_t c = P.at(qp, qn), d = P.at(qpp, qnn);
            const int sc = P.pair_sec[c - 1];
            if (sc != P.pair_sec[d - 1]) return 0.0;
            const int64_t first = P.sec_first[sc], n = P.sec_n[sc];
            return B.vpn[P.sec_mestart[sc] + (c - first) * n + (d - first + 1) - 1];
        };
        auto bit = [](int q) { return 1ull << q; };
        // <T| V_xx |T'> between three-particle states of one species
        auto v3xxx = [&](int it, const std::array<int, 3> &T, const std::array<int, 3> &U) -> double {
            const Pairs &P = it == 0 ? B.ppairs : B.npairs;
            const uint64_t bu = bit(U[0]) | bit(U[1]) | bit(U[2]);
            const uint64_t bt = bit(T[0]) | bit(T[1]) | bit(T[2]);
            double v = 0.0;
            for (int z : U) {
                if (!(bt >> z & 1ull)) continue;     // spectator z in both
                int x = -1, y = -1, i = -1, j = -1;
                for (int q : U) if (q != z) { if (x < 0) x = q; else y = q; }
                for (int q : T) if (q != z) { if (i < 0) i = q; else j = q; }
                v += vxx(it, P.at(i, j), P.at(x, y)) * phase2(bu, i, j, x, y);
            }
            return v;
        };
        // <(XX pair bb, y a)| V |(XX pair dd, y c)>: V_xx on the pair with y a
        // spectator, plus V_pn moving one X particle and the y particle
        auto v3xxy = [&](int itx, int bb, int a, int dd, int c) -> double {
            const Pairs &P = itx == 0 ? B.ppairs : B.npairs;
            double v = (a == c) ? vxx(itx, bb, dd) : 0.0;
            const int i = P.list[bb - 1].first, j = P.list[bb - 1].second;
            const int l = P.list[dd - 1].first, m = P.list[dd - 1].second;
            const uint64_t bd = bit(l) | bit(m), bc = bit(i) | bit(j);
            for (int pd : {l, m}) {
                const int z = (pd == l) ? m : l;     // X spectator
                if (!(bc >> z & 1ull)) continue;
                const int pc = (z == i) ? j : i;
                const double x = itx == 0 ? vpn(pc, a, pd, c) : vpn(a, pc, c, pd);
                if (x != 0.0) v += x * phase1(bd, pc, pd);
            }
            return v;
        };
        // ---- matrix elements: triangle sections (XXX), square sections (XXY)
        auto fill_xxx = [&](int it, const Trips &T, std::vector<float> &H) {
            H.assign(T.nmat, 0.0f);
            const int kind = it == 0 ? 1 : 2;
            for (size_t sc = 0; sc < T.sec_n.size(); ++sc) {
                const int64_t first = T.sec_first[sc], n = T.sec_n[sc];
                for (int64_t c = first; c < first + n; ++c)
                    for (int64_t d = first; d <= c; ++d) {
                        const auto &tc = T.list[c - 1], &td = T.list[d - 1];
                        double w = w2 * v3xxx(it, tc, td) + w3 * r3(seed, kind, tc, td);
                        if (c == d) w *= 0.5;    // applied by both 'f' and 'b'
                        H[xxx_label(T, c, d) - 1] = (float)w;
                    }
            }
        };
        auto fill_xxy = [&](int itx, const Trips &T, std::vector<float> &H, std::vector<int32_t> &ct,
                            std::vector<int32_t> &dt) {
            const SpeciesBasis &sy = itx == 0 ? B.nb : B.pb;
            const Pairs &P = itx == 0 ? B.ppairs : B.npairs;
            const int64_t npr = (int64_t)P.list.size(), ldy = sy.nl + sy.nr + 1;
            H.assign(T.nmat, 0.0f);
            ct.assign((size_t)(npr * ldy), -1);
            dt.assign((size_t)(npr * ldy), -1);
            const int kind = itx == 0 ? 3 : 4;
            auto key = [&](const std::array<int, 3> &t) -> std::array<int, 3> {
                const auto &pr = P.list[t[0] - 1];
                return itx == 0 ? std::array<int, 3>{pr.first, pr.second, t[1]}
                                : std::array<int, 3>{t[1], pr.first, pr.second};
            };
            for (size_t sc = 0; sc < T.sec_n.size(); ++sc) {
                const int64_t first = T.sec_first[sc], n = T.sec_n[sc], nme = T.sec_mestart[sc];
                for (int64_t pos = 1; pos <= n; ++pos) {
                    const auto &t = T.list[first + pos - 2];
                    const int64_t at = (int64_t)(t[0] - 1) + (int64_t)(signed_label(sy, t[1]) + sy.nl) * npr;
                    ct[at] = (int32_t)(nme + (pos - 1) * n);
                    dt[at] = (int32_t)pos;
                }
                for (int64_t cp = 1; cp <= n; ++cp)
                    for (int64_t dp = 1; dp <= n; ++dp) {
                        const auto &tc = T.list[first + cp - 2], &td = T.list[first + dp - 2];
                        double w = w2 * v3xxy(itx, tc[0], tc[1], td[0], td[1]) + w3 * r3(seed, kind, key(tc), key(td));
                        if (tc[0] == td[0]) w *= 0.5;   // equal pairs: the X jump is diagonal
                        H[nme + (cp - 1) * n + dp - 1] = (float)w;
                    }
            }
        };
        fill_xxx(0, Tppp, B.hmatppp);
        fill_xxx(1, Tnnn, B.hmatnnn);
        fill_xxy(0, Tppn, B.hmatppn, B.cppn, B.dppn);
        fill_xxy(1, Tpnn, B.hmatpnn, B.cpnn, B.dpnn);

        // ---- three-body jumps inside a sector (weld3b,
        // src/bjumplib_weld.f90:819-1208): SD, destroyed triplet, created
        // triplet of the same section; isd >= fsd
        auto gen3 = [&](SpeciesBasis &sb, const std::vector<int64_t> &xstart, const Trips &T, int is, Jumps2 &J) {
            int64_t cnt = 0;
            const Sector &S = sb.sectors[is];
            const int ns = sb.nl + sb.nr;
            std::vector<int> occ;
            for (int64_t sd = S.xsdstart - 1; sd < S.xsdend; ++sd) {
                const uint64_t bits = sb.sd_bits[sd];
                occ.clear();
                for (int q = 0; q < ns; ++q)
                    if (bits >> q & 1ull) occ.push_back(q);
                for (size_t x = 0; x < occ.size(); ++x)
                    for (size_t y = x + 1; y < occ.size(); ++y)
                        for (size_t z = y + 1; z < occ.size(); ++z) {
                            const int l = occ[x], m = occ[y], n = occ[z];
                            const uint64_t rest = bits & ~(bit(l) | bit(m) | bit(n));
                            const int64_t d = T.dense[colex3(l, m, n)];
                            for (int32_t c : T.by_sec[T.sec[d - 1]]) {
                                const auto &tc = T.list[c - 1];
                                if ((rest >> tc[0] & 1ull) || (rest >> tc[1] & 1ull) || (rest >> tc[2] & 1ull)) continue;
                                const int64_t f = sb.find_sd(rest | bit(tc[0]) | bit(tc[1]) | bit(tc[2]));
                                if (f < 0 || sb.sd_sector[f] != is) continue;
                                if (sd < f) continue;
                                J.isd.push_back(xstart[sd]);
                                J.fsd.push_back(xstart[f]);
                                J.op.push_back((int32_t)xxx_label(T, c, d));
                                J.phase.push_back((int8_t)phase3(bits, tc[0], tc[1], tc[2], l, m, n));
                                ++cnt;
                            }
                        }
            }
            return cnt;
        };
        // ---- two-body jumps with pair labels out of one sector, bucketed by
        // final sector (SD, destroyed pair, created pair); the diagonal bucket
        // keeps isd >= fsd
        std::map<std::pair<const SpeciesBasis *, int>, std::vector<Jumps2P>> jumps2_from;
        auto gen2x = [&](SpeciesBasis &sb, const std::vector<int64_t> &xstart, const Pairs &P, int is, int fs,
                         Jumps2P &J) -> int64_t {
            auto k = std::make_pair((const SpeciesBasis *)&sb, is);
            auto it = jumps2_from.find(k);
            if (it == jumps2_from.end()) {
                std::vector<Jumps2P> by(sb.sectors.size());
                const Sector &S = sb.sectors[is];
                const int ns = sb.nl + sb.nr;
                std::vector<int> occ;
                for (int64_t sd = S.xsdstart - 1; sd < S.xsdend; ++sd) {
                    const uint64_t bits = sb.sd_bits[sd];
                    occ.clear();
                    for (int q = 0; q < ns; ++q)
                        if (bits >> q & 1ull) occ.push_back(q);
                    for (size_t x = 0; x < occ.size(); ++x)
                        for (size_t y = x + 1; y < occ.size(); ++y) {
                            const int kq = occ[x], lq = occ[y];
                            const uint64_t rest = bits & ~(bit(kq) | bit(lq));
                            const int64_t dpair = P.at(kq, lq);
                            for (size_t c = 1; c <= P.list.size(); ++c) {
                                const int i = P.list[c - 1].first, j = P.list[c - 1].second;
                                if ((rest >> i & 1ull) || (rest >> j & 1ull)) continue;
                                const int64_t f = sb.find_sd(rest | bit(i) | bit(j));
                                if (f < 0) continue;
                                const int fsec = sb.sd_sector[f];
                                if (fsec == is && sd < f) continue;
                                Jumps2P &Bk = by[fsec];
                                Bk.isd.push_back(xstart[sd]);
                                Bk.fsd.push_back(xstart[f]);
                                Bk.cop.push_back((int32_t)c);
                                Bk.dop.push_back((int32_t)dpair);
                                Bk.phase.push_back((int8_t)phase2(bits, i, j, kq, lq));
                            }
                        }
                }
                it = jumps2_from.emplace(k, std::move(by)).first;
            }
            const Jumps2P &src = it->second[fs];
            J.isd.insert(J.isd.end(), src.isd.begin(), src.isd.end());
            J.fsd.insert(J.fsd.end(), src.fsd.begin(), src.fsd.end());
            J.cop.insert(J.cop.end(), src.cop.begin(), src.cop.end());
            J.dop.insert(J.dop.end(), src.dop.begin(), src.dop.end());
            J.phase.insert(J.phase.end(), src.phase.begin(), src.phase.end());
            return (int64_t)src.isd.size();
        };
        if (s->np >= 3)
            for (int is = 0; is < nps; ++is) {
                SectJump sj{is, is, (int64_t)B.p3.isd.size(), 0, true};
                sj.njumps = gen3(B.pb, B.pstart, Tppp, is, B.p3);
                if (sj.njumps > 0) p3sj.push_back(sj);
            }
        if (s->nn >= 3)
            for (int in = 0; in < nns; ++in) {
                SectJump sj{in, in, (int64_t)B.n3.isd.size(), 0, true};
                sj.njumps = gen3(B.nb, B.nstart, Tnnn, in, B.n3);
                if (sj.njumps > 0) n3sj.push_back(sj);
            }
        // PPN: proton two-body sector jumps is -> fs (is >= fs) with the
        // conjugate neutron one-body sector jump
        if (s->np >= 2 && s->nn >= 1)
            for (int is = 0; is < nps; ++is)
                for (int fs = 0; fs <= is; ++fs) {
                    Jumps2P tmp;
                    if (gen2x(B.pb, B.pstart, B.ppairs, is, fs, tmp) == 0) continue;
                    const int in = pconj[is], fn = pconj[fs];
                    int y;
                    if (n1sj_of.count({in, fn})) {
                        y = n1sj_of[{in, fn}];
                    } else {
                        SectJump nj{in, fn, (int64_t)B.n1.isd.size(), 0, in == fn};
                        nj.njumps = gen1(B.nb, B.nstart, in, fn, B.n1);
                        y = (int)B.n1sj.size();
                        n1sj_of[{in, fn}] = y;
                        B.n1sj.push_back(nj);
                    }
                    if (B.n1sj[y].njumps == 0) continue;
                    SectJump sj{is, fs, (int64_t)B.p2x.isd.size(), (int64_t)tmp.isd.size(), is == fs};
                    B.p2x.isd.insert(B.p2x.isd.end(), tmp.isd.begin(), tmp.isd.end());
                    B.p2x.fsd.insert(B.p2x.fsd.end(), tmp.fsd.begin(), tmp.fsd.end());
                    B.p2x.cop.insert(B.p2x.cop.end(), tmp.cop.begin(), tmp.cop.end());
                    B.p2x.dop.insert(B.p2x.dop.end(), tmp.dop.begin(), tmp.dop.end());
                    B.p2x.phase.insert(B.p2x.phase.end(), tmp.phase.begin(), tmp.phase.end());
                    p2xsj.push_back(sj);
                    p2x_n1.push_back(y);
                }
        // PNN: proton one-body sector jumps (those of the PN set-up) with the
        // conjugate neutron two-body sector jump
        if (s->np >= 1 && s->nn >= 2) {
            std::map<std::pair<int, int>, int> n2x_of;
            for (size_t x = 0; x < B.p1sj.size(); ++x) {
                const int in = pconj[B.p1sj[x].is], fn = pconj[B.p1sj[x].fs];
                int y;
                if (n2x_of.count({in, fn})) {
                    y = n2x_of[{in, fn}];
                } else {
                    SectJump nj{in, fn, (int64_t)B.n2x.isd.size(), 0, in == fn};
                    nj.njumps = gen2x(B.nb, B.nstart, B.npairs, in, fn, B.n2x);
                    y = (int)n2xsj.size();
                    n2x_of[{in, fn}] = y;
                    n2xsj.push_back(nj);
                }
                if (n2xsj[y].njumps == 0) continue;
                pnn_p1.push_back((int)x);
                pnn_n2x.push_back(y);
            }
        }
        B.t3.npairs_p = (int32_t)B.ppairs.list.size();
        B.t3.npairs_n = (int32_t)B.npairs.list.size();
    }

    // ---- one-body density jumps (set1bsectorjumps + master1bodyjumps for
    // densities, src/bdenslib1.f90:190-213): every sector jump is -> fs
    // (is >= fs) that keeps Jz, parity and the conjugate sector, all
    // a+_i a_k with i, k of equal m, a+_k a_k included.  A proton jump range
    // is paired with the conjugate neutron SDs (P1B), a neutron jump range
    // with the conjugate proton SDs (N1B); is > fs also gets a 'b' bundle,
    // which covers the reverse direction through the same jumps.
    {
        auto dadd = [&](int op, int hc, int64_t px0, int64_t px1, int64_t nx0, int64_t nx1) {
            B.d_optype.push_back(op); B.d_hchar.push_back(hc);
            B.d_pxstart.push_back(px0); B.d_pxend.push_back(px1);
            B.d_nxstart.push_back(nx0); B.d_nxend.push_back(nx1);
            B.d_cstride.push_back(1);
        };
        auto same_kind = [&](const SpeciesBasis &sb, int a, int b) {
            return sb.sectors[a].jz2 == sb.sectors[b].jz2 && sb.sectors[a].pidx == sb.sectors[b].pidx;
        };
        if (s->np >= 1)
            for (int is = 0; is < nps; ++is)
                for (int fs = 0; fs <= is; ++fs) {
                    if (!same_kind(B.pb, is, fs) || pconj[is] != pconj[fs]) continue;
                    const int64_t j0 = (int64_t)B.dp1.isd.size();
                    const int64_t nj = gen1(B.pb, B.pstart, is, fs, B.dp1);
                    if (nj == 0) continue;
                    const Sector &ns = B.nb.sectors[pconj[is]];
                    dadd(BSG_OP_P1B, BSG_H_FWD, j0 + 1, j0 + nj, ns.xsdstart, ns.xsdend);
                    if (is != fs) dadd(BSG_OP_P1B, BSG_H_BWD, j0 + 1, j0 + nj, ns.xsdstart, ns.xsdend);
                }
        // a proton SD combines with one neutron sector (no truncation), so
        // a neutron sector jump shares its conjugate protons only with itself
        if (s->nn >= 1)
            for (int in = 0; in < nns; ++in) {
                std::vector<int> psecs;
                for (int ip = 0; ip < nps; ++ip)
                    if (pconj[ip] == in) psecs.push_back(ip);
                if (psecs.empty()) continue;
                const int64_t j0 = (int64_t)B.dn1.isd.size();
                const int64_t nj = gen1(B.nb, B.nstart, in, in, B.dn1);
                if (nj == 0) continue;
                for (int ip : psecs) {
                    const Sector &ps = B.pb.sectors[ip];
                    dadd(BSG_OP_N1B, BSG_H_FWD, ps.xsdstart, ps.xsdend, j0 + 1, j0 + nj);
                }
            }
    }

    // ---- single-particle energies per SD when call_spe (makespeme)
    if (call_spe) {
        B.pspe_h.assign(nsdp, 0.0f);
        B.nspe_h.assign(nsdn, 0.0f);
        for (int it = 0; it < 2; ++it) {
            SpeciesBasis &sb = *sbs[it];
            auto &out = it == 0 ? B.pspe_h : B.nspe_h;
            for (size_t sd = 0; sd < sb.sd_bits.size(); ++sd) {
                double e = 0.0;
                for (int q = 0; q < sb.nl + sb.nr; ++q)
                    if (sb.sd_bits[sd] >> q & 1ull) e += spe[sb.q_orb[q]];
                out[sd] = (float)e;
            }
        }
    }

    // ---- opbundles in draft_opbundles order (src/bparallel_opbundles.f90:72-95)
    auto add = [&](int op, int hc, int64_t px0, int64_t px1, int64_t nx0, int64_t nx1) {
        B.optype.push_back(op); B.hchar.push_back(hc);
        B.pxstart.push_back(px0); B.pxend.push_back(px1);
        B.nxstart.push_back(nx0); B.nxend.push_back(nx1);
        B.cstride.push_back(1);
    };
    auto find_sj = [](const std::vector<SectJump> &v, int is, int fs) -> int {
        for (size_t i = 0; i < v.size(); ++i)
            if (v[i].is == is && v[i].fs == fs) return (int)i;
        return -1;
    };
    auto emit = [&](const char *kind, int hc) {
        for (int fs = 0; fs < nps; ++fs)
            for (int is = fs; is < nps; ++is) {
                if (!std::strcmp(kind, "PP")) {
                    const int x = find_sj(B.p2sj, is, fs);
                    if (x < 0) continue;
                    const Sector &ns = B.nb.sectors[pconj[is]];
                    add(BSG_OP_PP, hc, B.p2sj[x].nstart + 1, B.p2sj[x].nstart + B.p2sj[x].njumps, ns.xsdstart, ns.xsdend);
                } else if (!std::strcmp(kind, "NN")) {
                    if (is != fs) continue;
                    const int x = find_sj(B.n2sj, pconj[is], pconj[is]);
                    if (x < 0) continue;
                    const Sector &ps = B.pb.sectors[is];
                    add(BSG_OP_NN, hc, ps.xsdstart, ps.xsdend, B.n2sj[x].nstart + 1, B.n2sj[x].nstart + B.n2sj[x].njumps);
                } else {  // PN
                    const int x = find_sj(B.p1sj, is, fs);
                    if (x < 0) continue;
                    const int y = n1sj_of.count({pconj[is], pconj[fs]}) ? n1sj_of[{pconj[is], pconj[fs]}] : -1;
                    if (y < 0 || B.n1sj[y].njumps == 0) continue;
                    const bool herm = (is == fs && B.p1sj[x].diag && B.n1sj[y].diag);
                    if ((hc == BSG_H_HERM) != herm) continue;
                    add(BSG_OP_PN, hc, B.p1sj[x].nstart + 1, B.p1sj[x].nstart + B.p1sj[x].njumps,
                        B.n1sj[y].nstart + 1, B.n1sj[y].nstart + B.n1sj[y].njumps);
                }
            }
    };
    if (call_spe)
        for (int is = 0; is < nps; ++is) {
            const Sector &ps = B.pb.sectors[is];
            const Sector &ns = B.nb.sectors[pconj[is]];
            add(BSG_OP_SPE, BSG_H_HERM, ps.xsdstart, ps.xsdend, ns.xsdstart, ns.xsdend);
        }
    if (!three) {
        emit("PP", BSG_H_FWD);
        emit("NN", BSG_H_FWD);
        emit("PN", BSG_H_FWD);
        emit("PN", BSG_H_HERM);
        emit("PP", BSG_H_BWD);
        emit("NN", BSG_H_BWD);
        emit("PN", BSG_H_BWD);
    } else {
        // applyHbundled_g's three-body order (src/bapplyhlib1.f90:160-235):
        // PPP f/b, PPN f/b, PNN f/b, NNN f/b
        for (int hc : {BSG_H_FWD, BSG_H_BWD})
            for (const SectJump &sj : p3sj) {
                const Sector &ns = B.nb.sectors[pconj[sj.is]];
                add(BSG_OP_PPP, hc, sj.nstart + 1, sj.nstart + sj.njumps, ns.xsdstart, ns.xsdend);
            }
        for (int hc : {BSG_H_FWD, BSG_H_BWD})
            for (size_t x = 0; x < p2xsj.size(); ++x) {
                const SectJump &nj = B.n1sj[p2x_n1[x]];
                add(BSG_OP_PPN, hc, p2xsj[x].nstart + 1, p2xsj[x].nstart + p2xsj[x].njumps, nj.nstart + 1,
                    nj.nstart + nj.njumps);
            }
        for (int hc : {BSG_H_FWD, BSG_H_BWD})
            for (size_t x = 0; x < pnn_p1.size(); ++x) {
                const SectJump &pj = B.p1sj[pnn_p1[x]], &nj = n2xsj[pnn_n2x[x]];
                add(BSG_OP_PNN, hc, pj.nstart + 1, pj.nstart + pj.njumps, nj.nstart + 1, nj.nstart + nj.njumps);
            }
        for (int hc : {BSG_H_FWD, BSG_H_BWD})
            for (int is = 0; is < nps; ++is)
                for (const SectJump &nj : n3sj) {
                    if (nj.is != pconj[is]) continue;
                    const Sector &ps = B.pb.sectors[is];
                    add(BSG_OP_NNN, hc, ps.xsdstart, ps.xsdend, nj.nstart + 1, nj.nstart + nj.njumps);
                }
    }

    // ---- sort_bundled_jumps (src/bsortjumpslib.f90:21-175): per PN bundle,
    // protons on fsd, neutrons on isd
    // The 'f', 'h' and 'b' bundles of a sector jump share its ranges, and the
    // sort leaves a sorted range as it is, so each distinct range is sorted
    // once; the ranges of different sector jumps are disjoint, so they are
    // sorted on host threads.
    {
        std::vector<std::pair<int64_t, int64_t>> pr, nr;   // (0-based start, length)
        for (size_t ib = 0; ib < B.optype.size(); ++ib) {
            if (B.optype[ib] != BSG_OP_PN) continue;
            pr.push_back({B.pxstart[ib] - 1, B.pxend[ib] - B.pxstart[ib] + 1});
            nr.push_back({B.nxstart[ib] - 1, B.nxend[ib] - B.nxstart[ib] + 1});
        }
        for (auto *v : {&pr, &nr}) {
            std::sort(v->begin(), v->end());
            v->erase(std::unique(v->begin(), v->end()), v->end());
        }
        parallel_for((int64_t)(pr.size() + nr.size()), [&](int64_t j) {
            if (j < (int64_t)pr.size()) {
                const int64_t sp0 = pr[j].first, np_ = pr[j].second;
                shell_sort_1b(np_, B.p1.isd.data() + sp0, B.p1.fsd.data() + sp0, B.p1.cop.data() + sp0,
                              B.p1.dop.data() + sp0, B.p1.phase.data() + sp0);
            } else {
                const int64_t sn0 = nr[j - pr.size()].first, nn_ = nr[j - pr.size()].second;
                shell_sort_1b(nn_, B.n1.fsd.data() + sn0, B.n1.isd.data() + sn0, B.n1.cop.data() + sn0,
                              B.n1.dop.data() + sn0, B.n1.phase.data() + sn0);
            }
        });
    }

    // ---- sector / s.p. bookkeeping for the caller
    for (auto &sec : B.pb.sectors) {
        B.ps_start.push_back(sec.xsdstart); B.ps_end.push_back(sec.xsdend);
        B.ps_jz.push_back(sec.jz2); B.ps_par.push_back(par_of_idx(sec.pidx));
    }
    for (int a = 0; a < nps; ++a) B.ps_conj.push_back(pconj[a] + 1);
    for (auto &sec : B.nb.sectors) {
        B.ns_start.push_back(sec.xsdstart); B.ns_end.push_back(sec.xsdend);
        B.ns_jz.push_back(sec.jz2); B.ns_par.push_back(par_of_idx(sec.pidx));
    }
    for (int q = 0; q < B.pb.nl + B.pb.nr; ++q) { B.spo_p.push_back(B.pb.q_orb[q]); B.spm_p.push_back(B.pb.q_m2[q]); }
    for (int q = 0; q < B.nb.nl + B.nb.nr; ++q) { B.spo_n.push_back(B.nb.q_orb[q]); B.spm_n.push_back(B.nb.q_m2[q]); }
    (void)dimbasis;
    return BSG_OK;
}

template <typename T>
const T *ptr_or_null(const std::vector<T> &v) { return v.empty() ? nullptr : v.data(); }

}  // namespace

extern "C" {

const char *bsg_host_last_error(void) { return g_err.c_str(); }

int bsg_host_build(const bsg_model_spec *spec, bsg_host_tables **out) { return bsg_host_build3(spec, nullptr, out); }

int bsg_host_build3(const bsg_model_spec *spec, const bsg_model3_spec *s3, bsg_host_tables **out) {
    if (!out) { g_err = "null output"; return BSG_ERR_ARG; }
    *out = nullptr;
    Built *B = new (std::nothrow) Built();
    if (!B) { g_err = "host allocation failed"; return BSG_ERR_NOMEM; }
    int st;
    try {
        st = build(spec, s3, *B);
    } catch (const std::bad_alloc &) {
        g_err = "host allocation failed";
        st = BSG_ERR_NOMEM;
    } catch (const std::exception &e) {
        g_err = std::string("builder exception: ") + e.what();
        st = BSG_ERR_BAD_TABLE;
    }
    if (st != BSG_OK) { delete B; return st; }
    bsg_host_tables *h = (bsg_host_tables *)std::calloc(1, sizeof(bsg_host_tables));
    if (!h) { delete B; g_err = "host allocation failed"; return BSG_ERR_NOMEM; }
    bsg_tables &t = h->t;
    t.nsd_p = (int64_t)B->pstart.size();
    t.nsd_n = (int64_t)B->nstart.size();
    {
        int64_t dim = 0;
        for (size_t is = 0; is < B->ps_start.size(); ++is) {
            const int64_t pd = B->ps_end[is] - B->ps_start[is] + 1;
            const int c = B->ps_conj[is] - 1;
            dim += pd * (B->ns_end[c] - B->ns_start[c] + 1);
        }
        t.dimbasis = dim;
    }
    t.pstart = ptr_or_null(B->pstart);
    t.nstart = ptr_or_null(B->nstart);
    t.np1b = (int64_t)B->p1.isd.size();
    t.p1b_isd = ptr_or_null(B->p1.isd); t.p1b_fsd = ptr_or_null(B->p1.fsd);
    t.p1b_cop = ptr_or_null(B->p1.cop); t.p1b_dop = ptr_or_null(B->p1.dop); t.p1b_phase = ptr_or_null(B->p1.phase);
    t.nn1b = (int64_t)B->n1.isd.size();
    t.n1b_isd = ptr_or_null(B->n1.isd); t.n1b_fsd = ptr_or_null(B->n1.fsd);
    t.n1b_cop = ptr_or_null(B->n1.cop); t.n1b_dop = ptr_or_null(B->n1.dop); t.n1b_phase = ptr_or_null(B->n1.phase);
    t.np2b = (int64_t)B->p2.isd.size();
    t.p2b_isd = ptr_or_null(B->p2.isd); t.p2b_fsd = ptr_or_null(B->p2.fsd);
    t.p2b_op = ptr_or_null(B->p2.op); t.p2b_phase = ptr_or_null(B->p2.phase);
    t.nn2b = (int64_t)B->n2.isd.size();
    t.n2b_isd = ptr_or_null(B->n2.isd); t.n2b_fsd = ptr_or_null(B->n2.fsd);
    t.n2b_op = ptr_or_null(B->n2.op); t.n2b_phase = ptr_or_null(B->n2.phase);
    t.nmatpp = (int64_t)B->hmatpp.size(); t.hmatpp = ptr_or_null(B->hmatpp);
    t.nmatnn = (int64_t)B->hmatnn.size(); t.hmatnn = ptr_or_null(B->hmatnn);
    t.nmatpn = (int64_t)B->hmatpn.size(); t.hmatpn = ptr_or_null(B->hmatpn);
    t.nhsps_pl = B->pb.nl; t.nhsps_pr = B->pb.nr;
    t.nhsps_nl = B->nb.nl; t.nhsps_nr = B->nb.nr;
    t.cpnpair = ptr_or_null(B->cpn); t.dpnpair = ptr_or_null(B->dpn);
    t.call_spe = B->pspe_h.empty() ? 0 : 1;
    t.pspe_h = ptr_or_null(B->pspe_h); t.nspe_h = ptr_or_null(B->nspe_h);
    t.nbundles = (int64_t)B->optype.size();
    t.optype = ptr_or_null(B->optype); t.hchar = ptr_or_null(B->hchar);
    t.pxstart = ptr_or_null(B->pxstart); t.pxend = ptr_or_null(B->pxend);
    t.nxstart = ptr_or_null(B->nxstart); t.nxend = ptr_or_null(B->nxend);
    t.cstride = ptr_or_null(B->cstride);
    h->nsectors_p = (int32_t)B->ps_start.size();
    h->nsectors_n = (int32_t)B->ns_start.size();
    h->psector_start = B->ps_start.data(); h->psector_end = B->ps_end.data();
    h->psector_jz2 = B->ps_jz.data(); h->psector_par = B->ps_par.data();
    h->nsector_start = B->ns_start.data(); h->nsector_end = B->ns_end.data();
    h->nsector_jz2 = B->ns_jz.data(); h->nsector_par = B->ns_par.data();
    h->psector_conj = B->ps_conj.data();
    h->nhsps_p = B->pb.nl + B->pb.nr;
    h->nhsps_n = B->nb.nl + B->nb.nr;
    h->sp_orb_p = B->spo_p.data(); h->sp_m2_p = B->spm_p.data();
    h->sp_orb_n = B->spo_n.data(); h->sp_m2_n = B->spm_n.data();
    h->sd_bits_p = B->pb.sd_bits.data(); h->sd_bits_n = B->nb.sd_bits.data();
    h->npairs_pp = (int64_t)B->ppairs.list.size();
    h->npairs_nn = (int64_t)B->npairs.list.size();
    h->npairs_pn = (int64_t)B->pnpairs.list.size();
    bsg_density_tables &d = h->dt;
    d.np1b = (int64_t)B->dp1.isd.size();
    d.p1b_isd = ptr_or_null(B->dp1.isd); d.p1b_fsd = ptr_or_null(B->dp1.fsd);
    d.p1b_cop = ptr_or_null(B->dp1.cop); d.p1b_dop = ptr_or_null(B->dp1.dop); d.p1b_phase = ptr_or_null(B->dp1.phase);
    d.nn1b = (int64_t)B->dn1.isd.size();
    d.n1b_isd = ptr_or_null(B->dn1.isd); d.n1b_fsd = ptr_or_null(B->dn1.fsd);
    d.n1b_cop = ptr_or_null(B->dn1.cop); d.n1b_dop = ptr_or_null(B->dn1.dop); d.n1b_phase = ptr_or_null(B->dn1.phase);
    d.nbundles = (int64_t)B->d_optype.size();
    d.optype = ptr_or_null(B->d_optype); d.hchar = ptr_or_null(B->d_hchar);
    d.pxstart = ptr_or_null(B->d_pxstart); d.pxend = ptr_or_null(B->d_pxend);
    d.nxstart = ptr_or_null(B->d_nxstart); d.nxend = ptr_or_null(B->d_nxend);
    d.cstride = ptr_or_null(B->d_cstride);
    if (B->three) {
        // two-body jumps carry pair labels (no p2b_op / n2b_op)
        t.np2b = (int64_t)B->p2x.isd.size();
        t.p2b_isd = ptr_or_null(B->p2x.isd); t.p2b_fsd = ptr_or_null(B->p2x.fsd);
        t.p2b_op = nullptr; t.p2b_phase = ptr_or_null(B->p2x.phase);
        t.nn2b = (int64_t)B->n2x.isd.size();
        t.n2b_isd = ptr_or_null(B->n2x.isd); t.n2b_fsd = ptr_or_null(B->n2x.fsd);
        t.n2b_op = nullptr; t.n2b_phase = ptr_or_null(B->n2x.phase);
        bsg_tables3 &u = B->t3;
        u.p2b_cop = ptr_or_null(B->p2x.cop); u.p2b_dop = ptr_or_null(B->p2x.dop);
        u.n2b_cop = ptr_or_null(B->n2x.cop); u.n2b_dop = ptr_or_null(B->n2x.dop);
        u.np3b = (int64_t)B->p3.isd.size();
        u.p3b_isd = ptr_or_null(B->p3.isd); u.p3b_fsd = ptr_or_null(B->p3.fsd);
        u.p3b_op = ptr_or_null(B->p3.op); u.p3b_phase = ptr_or_null(B->p3.phase);
        u.nn3b = (int64_t)B->n3.isd.size();
        u.n3b_isd = ptr_or_null(B->n3.isd); u.n3b_fsd = ptr_or_null(B->n3.fsd);
        u.n3b_op = ptr_or_null(B->n3.op); u.n3b_phase = ptr_or_null(B->n3.phase);
        u.nmatppp = (int64_t)B->hmatppp.size(); u.hmatppp = ptr_or_null(B->hmatppp);
        u.nmatnnn = (int64_t)B->hmatnnn.size(); u.hmatnnn = ptr_or_null(B->hmatnnn);
        u.nmatppn = (int64_t)B->hmatppn.size(); u.hmatppn = ptr_or_null(B->hmatppn);
        u.nmatpnn = (int64_t)B->hmatpnn.size(); u.hmatpnn = ptr_or_null(B->hmatpnn);
        u.cppntriplet = ptr_or_null(B->cppn); u.dppntriplet = ptr_or_null(B->dppn);
        u.cpnntriplet = ptr_or_null(B->cpnn); u.dpnntriplet = ptr_or_null(B->dpnn);
        h->t3 = &B->t3;
    }
    h->priv = B;
    *out = h;
    return BSG_OK;
}

void bsg_host_free(bsg_host_tables *h) {
    if (!h) return;
    delete (Built *)h->priv;
    std::free(h);
}

int bsg_host_me_jacobian(const bsg_host_tables *h, int kind, double *d_tbme, double *d_spe) {
    if (!h || !h->priv || kind < 0 || kind > 2) { g_err = "bad jacobian request"; return BSG_ERR_ARG; }
    const Built *B = (const Built *)h->priv;
    const auto &jac = kind == 0 ? B->jac_pp : kind == 1 ? B->jac_nn : B->jac_pn;
    const auto &jsp = kind == 0 ? B->jspe_pp : kind == 1 ? B->jspe_nn : B->jspe_pn;
    const size_t nmat = jac.size();
    if (d_tbme) {
        std::memset(d_tbme, 0, sizeof(double) * nmat * (size_t)std::max(1, B->ntbme));
        for (size_t k = 0; k < nmat; ++k)
            for (auto &p : jac[k]) d_tbme[k * (size_t)B->ntbme + p.first] += p.second;
    }
    if (d_spe) {
        std::memset(d_spe, 0, sizeof(double) * nmat * (size_t)B->norb);
        for (size_t k = 0; k < nmat; ++k)
            for (auto &p : jsp[k]) d_spe[k * (size_t)B->norb + p.first] += p.second;
    }
    return BSG_OK;
}

}  // extern "C"
