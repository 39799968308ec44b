// Internal declarations shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "bsg.h"

namespace bsg {

// warps per applyH CTA; each row's contributions are split over them
constexpr int kRowWarps = 8;

// ---- derived (device) layouts, built once at bsg_create from the unchanged
// tables.  Positions are 0-based neutron positions inside a proton-SD row
// (position = nstart - 1); a row's first basis state (0-based) is pstart(ip).

// PP row contribution: out[row][pos] += me * in[q_off + pos], pos in [lo, hi]
struct PPContrib {
    int64_t q_off;
    float me;        // hmatpp(op) * phase, rounded to float as the reference
    int32_t lo, hi;
    int32_t pad;
};
// PN row contribution: out[row][pos] += sum over neutron-op records r at pos of
//   hmat(cpn[r.b + aoff] + dpn[r.d + coff]) * php * r.ph * in[q_off + r.in]
// The same form carries the three-body PPN and PNN terms: cpn / dpn / hmat
// on the device are the concatenation of the PN, PPN and PNN tables, and
// aoff / coff select the column of the proton side's label in its table
// (PN: proton s.p. a; PPN: proton pair bb; PNN: proton s.p. a with the
// neutron pair as the row).
struct PNContrib {
    int64_t q_off;
    int32_t nop;       // neutron operator id
    int32_t aoff;      // column offset of the created proton label in cpn
    int32_t coff;      // column offset of the destroyed proton label in dpn
    float php;         // proton jump phase
};
// NN row contribution: out[row][pos] += sum over records r at pos of r.me * in[row + r.in]
struct NNContrib {
    int32_t nop;
};
// SPE row contribution: out[row][pos] += (pspe + nspe[n0 + pos - lo]) * in[row + pos]
struct SPEContrib {
    float pspe;
    int32_t lo, hi;
    int32_t n0;       // 0-based neutron SD index at pos == lo
};
// neutron operator: records sorted by output position
struct NOp {
    int64_t rec_base;   // first record
    int64_t ptr_base;   // first entry of its [nout+1] pointer array
    int32_t nout;
    int32_t kind;       // 0 = NN (me records), 1 = PN (label records)
    int32_t bd_base;    // PN: first entry of its distinct (b,d) list
    int32_t nbd;        // PN: number of distinct (b,d) neutron label pairs
    // sliced copy of the records for the row kernels: output positions in
    // slices of 32; record k of position 32*s + l sits at
    // sell[sell_base + slice_off[slice_base + s] + 32*k + l], so the lanes of
    // a warp read adjacent records
    int64_t sell_base;
    int64_t slice_base;
};
// PN record: input position, index of its (b,d) pair in the operator's
// distinct-pair list, neutron jump phase
struct PNRec {
    int32_t in;
    uint16_t k;         // (b,d) pair = bd_list[bd_base + k]
    int8_t ph;
    int8_t pad;
};
// distinct (b,d) label pair of a PN neutron operator: rows of the cpn/dpn
// tables (a neutron s.p. label b + nhsps(-2), or for PNN a neutron pair - 1)
struct BDPair {
    uint16_t b, d;
};
// NN record: input position and hmatnn(op)*phase
struct NNRec {
    int32_t in;
    float me;
};
struct Tile {
    int32_t row;
    int32_t pos0;
    int32_t npos;
    int32_t pad;
};

struct RowArgs {
    const int64_t *row_off;       // [nrows] pstart
    const int32_t *pp_ptr, *nn_ptr, *pn_ptr, *spe_ptr;  // [nrows*kRowWarps+1] (row, warp) slots
    const PPContrib *pp;
    const NNContrib *nn;
    const PNContrib *pn;
    const SPEContrib *spe;
    const NOp *nops;
    const int32_t *nptr;          // pointer arrays of all neutron ops
    const PNRec *pnrec;
    const NNRec *nnrec;
    const int2 *sell;             // sliced PN / NN records (see NOp)
    // the same sliced records packed into 32 bits (null when a position or a
    // label does not fit): bits 0-15 input position, 16-30 the PN (b,d)
    // index or the NN hmatnn label - 1, bit 31 the jump phase's sign
    const uint32_t *sell32;
    const float *hmatnn;          // hmatnn (1-based labels; the NN 32-bit records index it)
    const int32_t *slice_off;
    const BDPair *bd;
    const float *hmatpn;
    const int32_t *cpn, *dpn;     // cpnpair/dpnpair as int32 (validated)
    const float *nspe;
    int32_t ld_cpn;               // nhsps(-2)+nhsps(2)+1
    int32_t ncpn;                 // entries of cpn
    int32_t max_nbd;              // largest nbd of any PN operator
    const Tile *tiles;
    int32_t ntiles;
    int32_t accumulate;
    // optional: store the result as FP64 columns (column v at cols_out +
    // v * cols_ld) instead of the interleaved output vector; the Lanczos
    // history takes it directly
    double *cols_out;
    int64_t cols_ld;
};

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

struct TileSet {
    DevBuf buf;
    int32_t ntiles = 0;
};

// row tiles cut into row-range chunks (host-pointer applyH copies each
// chunk's output out while the next chunks run): one owned buffer, chunk c's
// tiles at [start[c], start[c+1]) in longest-processing-time order, its
// states [s0[c], s0[c+1]); view[c] points into the buffer (not owned)
struct ChunkTiles {
    DevBuf buf;
    std::vector<int32_t> start;
    std::vector<int64_t> s0;
    std::vector<TileSet> view;
};

}  // namespace bsg

struct bsg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    int last_status = 0;      // status of the last set_err
    bool threebody = false;   // built by bsg_create3 (SPE + PPP/NNN/PPN/PNN)
    bool rec32_nn = false;    // the 32-bit records hold NN labels too (FP64 reads them)
    bsg_tables t{};           // sizes only (pointers are host-owned by caller)
    int64_t dim = 0, nrows = 0;
    int32_t max_rowlen = 0;
    int32_t median_rowlen = 0;
    int32_t max_nb = 16;
    int32_t pn_table_max = 512;   // bsg_config.pn_table_max
    // raw tables on the device (byte-identical copies)
    std::vector<bsg::DevBuf> raw;
    // derived
    bsg::DevBuf row_off, pp_ptr, nn_ptr, pn_ptr, spe_ptr, pp, nn, pn, spe, nops, nptr, pnrec, nnrec, bd, sell, slice_off;
    bsg::DevBuf sell32;
    bsg::DevBuf hmatpn, cpn, dpn, nspe, hmatpp_d, hmatnn_d;
    bsg::RowArgs args{};
    std::map<int, bsg::TileSet> tiles;   // tile size -> tiles
    // largest dynamic shared memory already allowed per kernel function (the
    // attribute is set once per size, not on every launch)
    std::map<const void *, size_t> smem_allowed;
    std::vector<int32_t> h_rowlen;
    std::vector<bsg::BDPair> h_bd;
    std::vector<bsg::PNRec> h_pnrec;
    std::vector<int32_t> h_nptr;
    std::vector<int32_t> h_work;         // per-row work estimate
    // host copies kept for the adjoint
    std::vector<int32_t> h_pp_ptr, h_nn_ptr, h_pn_ptr;
    std::vector<bsg::PPContrib> h_pp;
    std::vector<int32_t> h_pp_op;        // hmatpp label of each PP contribution
    std::vector<int8_t> h_pp_ph;         // jump phase of each PP contribution
    std::vector<bsg::NNContrib> h_nn;
    std::vector<bsg::PNContrib> h_pn;
    std::vector<bsg::NOp> h_nops;
    std::vector<int32_t> h_nnrec_op;     // hmatnn label of each NN record
    bsg::DevBuf pp_op, nnrec_op, nnrec_ph, pp_ph;
    bsg_stats stats{};
    // scratch vectors for host-pointer applyh
    bsg::DevBuf scratch_in, scratch_out;
    // chunked host-pointer applyh: tiles per tile size, the copy stream and
    // one event per chunk
    std::map<int, bsg::ChunkTiles> chunk_tiles;
    cudaStream_t copy_stream = nullptr;
    std::vector<cudaEvent_t> chunk_ev;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace bsg {
int set_err(bsg_ctx *ctx, int code, const std::string &msg);
int cuda_check(bsg_ctx *ctx, cudaError_t e, const char *what);
int dev_alloc(bsg_ctx *ctx, DevBuf &b, size_t bytes);
void dev_free(DevBuf &b);
int upload(bsg_ctx *ctx, DevBuf &b, const void *src, size_t bytes);
const TileSet *get_tiles(bsg_ctx *ctx, int tp);
// row tiles of width tp in longest-processing-time order (host list)
void build_tile_list(const bsg_ctx *ctx, int tp, std::vector<Tile> &tiles);
// where applyH finds its row tiles; nullptr = the context's own (built and
// cached on first use)
typedef const TileSet *(*TileLookup)(bsg_ctx *ctx, int tp);
int launch_applyh(bsg_ctx *ctx, const void *vin, void *vout, int nb, int prec, int accumulate,
                  cudaStream_t s, TileLookup lookup = nullptr);
// H x for an interleaved input x (nb <= 16, dense and 16-byte aligned), the
// result written as nb FP64 columns of length dim starting at cols
int launch_applyh_cols(bsg_ctx *ctx, const void *vin, double *cols, int nb, int prec, cudaStream_t s);
// adjoint gradients of nsys systems x nstates states in one launch
// (grad.cu); evecs[s] host dim_s x nstates column-major; outputs host
// [state][label] per system (dspe_* may be null); kernel_ms: device time
int grad_many(bsg_ctx *const *ctxs, int nsys, const double *const *evecs, int nstates, double *const *dpp,
              double *const *dnn, double *const *dpn, double *const *dspe_p, double *const *dspe_n, cudaStream_t s,
              std::string &err, double *kernel_ms);
}  // namespace bsg
