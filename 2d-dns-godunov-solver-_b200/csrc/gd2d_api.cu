// Host side of the C ABI declared in include/godunov2d.h.
//
// gd2d_setup validates the reference-layout meshes, reorders cells and
// nodes along a Hilbert curve (or keeps the natural order), concatenates
// all cases with per-case padding so that no tile of the cell kernel spans
// two cases, and uploads the packed layout.  The permutation is kept with
// its exact inverse so that every download is in reference order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/godunov2d.h"
#include "gd2d_internal.h"

using namespace gd2d;

namespace {

thread_local std::string g_setup_error;

struct HostCase {
    int64_t nc = 0, nn = 0, nc_pad = 0;
    int64_t cell_off = 0, node_off = 0;
    int64_t ref_off = 0, nref_off = 0;        // offsets in the compact reference-order index arrays
    std::vector<int64_t> cell_perm, cell_inv;  // perm[new] = old, inv[old] = new
    std::vector<int64_t> node_perm, node_inv;
    gd2d_params params{};
    double start_time = 0.0;
    bool state_set = false;
};

struct DevBuffers {
    std::vector<void *> all;
    template <class T>
    cudaError_t alloc(T **p, size_t count) {
        *p = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
        if (e == cudaSuccess) {
            all.push_back(*p);
            e = cudaMemset(*p, 0, count * sizeof(T));
        }
        return e;
    }
    void free_all() {
        for (void *p : all) cudaFree(p);
        all.clear();
    }
};

// Host worker threads of a handle's staged transfers, started on first use
// and kept until the handle is destroyed, so that a transfer does not pay
// the start-up of its threads (tens of microseconds each).  run() hands out
// items 0..n-1 in increasing order to the workers and the calling thread and
// returns once every item is done.
class StagePool {
  public:
    ~StagePool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            quit_ = true;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
    }
    void run(int device, unsigned workers, unsigned n, const std::function<void(unsigned)> &fn) {
        if (th_.size() < workers) start(device, workers);
        std::unique_lock<std::mutex> lk(mu_);
        job_ = &fn;
        njobs_ = n;
        next_ = 0;
        finished_ = 0;
        ++gen_;
        cv_.notify_all();
        drain(lk);
        done_cv_.wait(lk, [&] { return finished_ == njobs_; });
        job_ = nullptr;
    }

  private:
    void start(int device, unsigned workers) {
        while (th_.size() < workers) {
            th_.emplace_back([this, device] {
                cudaSetDevice(device);  // the DMAs are queued from these threads
                uint64_t seen = 0;
                std::unique_lock<std::mutex> lk(mu_);
                for (;;) {
                    cv_.wait(lk, [&] { return quit_ || (gen_ != seen && job_ != nullptr); });
                    if (quit_) return;
                    seen = gen_;
                    drain(lk);
                }
            });
        }
    }
    // Takes items until none is left (mu_ held on entry and exit).
    void drain(std::unique_lock<std::mutex> &lk) {
        while (job_ && next_ < njobs_) {
            const unsigned k = next_++;
            const std::function<void(unsigned)> *fn = job_;
            lk.unlock();
            (*fn)(k);
            lk.lock();
            if (++finished_ == njobs_) done_cv_.notify_all();
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(unsigned)> *job_ = nullptr;
    unsigned njobs_ = 0, next_ = 0, finished_ = 0;
    uint64_t gen_ = 0;
    bool quit_ = false;
};

}  // namespace

struct gd2d_handle {
    int device = 0;
    int32_t ncases = 0;
    std::vector<HostCase> cases;
    gd2d_launch launch{};
    LaunchCfg lc{};
    int flux = FLUX_AUSM;
    bool visc = false, quads = false, tgv = false, mixed = false;
    DevMesh m{};
    DevState s{};
    DevBuffers buf;
    std::vector<DevCase> hcases;
    std::vector<int32_t> tile_case_h;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaGraphExec_t graph = nullptr;
    cudaGraphExec_t graph1 = nullptr;  // one step, for the remainder of a propagate call
    int graph_steps = 0;
    bool state_ready = false;
    std::vector<std::vector<gd2d_stats>> history;
    std::vector<cudaEvent_t> ev;  // pairs around cell kernels of the captured graph
    cudaEvent_t ev_total[2] = {nullptr, nullptr};
    cudaEvent_t ev_eager[2] = {nullptr, nullptr};  // around the cell kernel of the last eager step
    double last_total_ms = 0.0, last_cell_ms = 0.0;
    int64_t last_launches = 0;
    // reordering between reference and device order, on the device
    int32_t *d_perm = nullptr;   // [Nc] reference row of each device cell
    int32_t *d_inv = nullptr;    // [sum nc] device cell of each reference row
    int32_t *d_ninv = nullptr;   // [sum nn] device node of each reference node
    double *d_stage = nullptr;   // [4 x max(nc, nn)] reference-order columns in transit
    double *h_stage = nullptr;   // page-locked host copy of d_stage
    // face-loop variants: faces sorted by colour, colour ranges, flux storage
    int loop = GD2D_LOOP_CELL;
    int4 *d_faces = nullptr;
    int64_t nfaces = 0;
    int64_t ngroups = 0;  // tile groups of the step reduction, all cases
    std::vector<int64_t> colour_off;
    double4 *Facc = nullptr, *Fslot = nullptr;
    // single-function entry points
    double4 *split_unew = nullptr, *split_flux = nullptr, *split_delta = nullptr, *split_diff = nullptr;
    bool split_stage_done = false, split_diff_valid = false;
    std::vector<CaseState> cs_host;  // host copy: steps taken per case (advanced by propagate)
    DevStats *ring_host = nullptr;    // page-locked, mapped copy of the statistics ring
    std::vector<cudaEvent_t> slice_ev;  // one per slice of a staged download
    StagePool pool;                     // host threads of the staged transfers
    std::string err;
};

namespace {

int fail(gd2d_handle *h, int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (h) h->err = buf;
    else g_setup_error = buf;
    return code;
}

#define CUDA_TRY(h, call)                                                                          \
    do {                                                                                           \
        cudaError_t e__ = (call);                                                                  \
        if (e__ != cudaSuccess)                                                                    \
            return fail((h), e__ == cudaErrorMemoryAllocation ? GD2D_ERR_OOM : GD2D_ERR_CUDA,      \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e__), __FILE__, __LINE__);     \
    } while (0)

inline int64_t cidx(int64_t n, int64_t i, int64_t j) { return i + j * n; }

// Hilbert index of (x, y) on a 2^16 grid (Butz / Lam-Shapiro iterative form).
uint64_t hilbert_index(uint32_t x, uint32_t y) {
    const uint32_t n = 1u << 16;
    uint64_t d = 0;
    for (uint32_t s = n / 2; s > 0; s /= 2) {
        uint32_t rx = (x & s) ? 1u : 0u;
        uint32_t ry = (y & s) ? 1u : 0u;
        d += (uint64_t)s * (uint64_t)s * (uint64_t)((3u * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) {
                x = n - 1 - x;
                y = n - 1 - y;
            }
            std::swap(x, y);
        }
    }
    return d;
}

void hilbert_order(const std::vector<double> &xs, const std::vector<double> &ys, std::vector<int64_t> &perm) {
    const size_t n = xs.size();
    double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY;
    for (size_t i = 0; i < n; ++i) {
        x0 = std::min(x0, xs[i]); x1 = std::max(x1, xs[i]);
        y0 = std::min(y0, ys[i]); y1 = std::max(y1, ys[i]);
    }
    double span = std::max(x1 - x0, y1 - y0);
    if (!(span > 0)) span = 1.0;
    std::vector<uint64_t> key(n);
    for (size_t i = 0; i < n; ++i) {
        uint32_t qx = (uint32_t)std::min(65535.0, std::floor((xs[i] - x0) / span * 65535.0));
        uint32_t qy = (uint32_t)std::min(65535.0, std::floor((ys[i] - y0) / span * 65535.0));
        key[i] = hilbert_index(qx, qy);
    }
    perm.resize(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
}

// Reverse Cuthill-McKee over the face-neighbour graph of the cells.
void rcm_order(const gd2d_mesh_view &mv, std::vector<int64_t> &perm) {
    const int64_t n = mv.n_cells;
    std::vector<int> deg(n, 0);
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < 4; ++k) if (mv.cell_stiffness[cidx(n, i, k)] >= 1) ++deg[i];
    std::vector<char> seen(n, 0);
    std::vector<int64_t> order;
    order.reserve(n);
    std::vector<int64_t> byd(n);
    std::iota(byd.begin(), byd.end(), 0);
    std::stable_sort(byd.begin(), byd.end(), [&](int64_t a, int64_t b) { return deg[a] < deg[b]; });
    for (int64_t s0 : byd) {
        if (seen[s0]) continue;
        size_t head = order.size();
        order.push_back(s0);
        seen[s0] = 1;
        while (head < order.size()) {
            int64_t i = order[head++];
            int64_t nb[4];
            int cnt = 0;
            for (int k = 0; k < 4; ++k) {
                int32_t st = mv.cell_stiffness[cidx(n, i, k)];
                if (st >= 1 && !seen[st - 1]) { nb[cnt++] = st - 1; seen[st - 1] = 1; }
            }
            std::sort(nb, nb + cnt, [&](int64_t a, int64_t b) { return deg[a] < deg[b]; });
            for (int q = 0; q < cnt; ++q) order.push_back(nb[q]);
        }
    }
    perm.assign(order.rbegin(), order.rend());
}

int validate_mesh(int c, const gd2d_mesh_view &mv, const gd2d_params &p) {
    const int64_t n = mv.n_cells, nn = mv.n_nodes;
    if (n <= 0 || nn <= 0) return fail(nullptr, GD2D_ERR_MESH, "case %d: empty mesh", c);
    if (n >= (1LL << 30) || nn >= (1LL << 30)) return fail(nullptr, GD2D_ERR_MESH, "case %d: mesh too large", c);
    if (!mv.mesh_connectivity || !mv.cell_stiffness || !mv.cell_edges_Nx || !mv.cell_edges_Ny ||
        !mv.cell_edges_length || !mv.cell_areas || !mv.HX || !mv.cell_clusters || !mv.node2cellL2up ||
        !mv.node2cellL2down || !mv.cells2nodes || !mv.cell_mid_points || !mv.x_nodes || !mv.y_nodes)
        return fail(nullptr, GD2D_ERR_ARG, "case %d: a mesh array pointer is NULL", c);
    if (mv.n_neib_cells < 1 || mv.n_neib_cells > 64)
        return fail(nullptr, GD2D_ERR_MESH, "case %d: n_neib_cells=%d out of range", c, mv.n_neib_cells);
    for (int64_t i = 0; i < n; ++i) {
        int32_t typ = mv.mesh_connectivity[cidx(n, i, 1)];
        int32_t nf = mv.mesh_connectivity[cidx(n, i, 2)];
        if (!((nf == 3 && typ == 3) || (nf == 4 && typ == 2)))
            return fail(nullptr, GD2D_ERR_MESH, "case %d: cell %lld has type %d with %d nodes", c, (long long)i + 1,
                        typ, nf);
        if (!(mv.cell_areas[i] > 0.0))
            return fail(nullptr, GD2D_ERR_MESH, "case %d: cell %lld has non-positive area", c, (long long)i + 1);
        for (int k = 0; k < nf; ++k) {
            int32_t st = mv.cell_stiffness[cidx(n, i, k)];
            if (st > n || st == 0)
                return fail(nullptr, GD2D_ERR_MESH, "case %d: cell %lld face %d neighbour %d out of range", c,
                            (long long)i + 1, k + 1, st);
            if (st < 0) {
                bool found = false;
                for (int b = 0; b < p.n_bc; ++b) found |= (p.bc[b].tag == st);
                if (!found)
                    return fail(nullptr, GD2D_ERR_MESH, "case %d: boundary tag %d has no entry in params.bc", c, st);
            } else {
                int idx = 2 * k;
                int cntn = (nf == 4) ? 2 : 1;
                for (int q = 0; q < cntn; ++q) {
                    int32_t d = mv.node2cellL2down[cidx(n, i, idx + q)], u = mv.node2cellL2up[cidx(n, i, idx + q)];
                    if (d < 1 || d > nn || u < 1 || u > nn)
                        return fail(nullptr, GD2D_ERR_MESH, "case %d: cell %lld face %d: up/down node out of range", c,
                                    (long long)i + 1, k + 1);
                }
            }
            for (int q = 0; q < 2; ++q) {
                int32_t e = mv.cells2nodes[cidx(n, i, 2 * k + q)];
                if (e < 1 || e > nn)
                    return fail(nullptr, GD2D_ERR_MESH, "case %d: cell %lld cells2nodes out of range", c,
                                (long long)i + 1);
            }
        }
    }
    for (int64_t J = 0; J < nn; ++J)
        for (int j = 0; j < mv.n_neib_cells; ++j) {
            int32_t cc = mv.cell_clusters[cidx(nn, J, j)];
            if (cc < 0 || cc > n)
                return fail(nullptr, GD2D_ERR_MESH, "case %d: node %lld cluster entry %d out of range", c,
                            (long long)J + 1, cc);
        }
    return GD2D_OK;
}

DevCase make_devcase(const gd2d_params &p, double maxEdge) {
    DevCase d{};
    d.gamma = p.Gamma;
    d.R = p.RGAS;
    d.CFL = p.CFL;
    d.dt_fixed = p.dt;
    d.beta = p.beta;
    d.ksi = p.ksi;
    d.venkat_K = p.venkat_K;
    d.mu_ref = p.mu_ref;
    d.suth_ref = 1.4792e-6 * std::sqrt(p.T_ref) / (1.0 + 116.0 / p.T_ref);
    d.gamma_over_Pr = p.Gamma / p.Pr;
    d.maxEdge = maxEdge;
    d.tgv_U0 = p.tgv_U0;
    d.tgv_P0 = p.tgv_P0;
    d.tgv_L = p.tgv_L;
    d.tgv_mu = p.tgv_mu;
    for (int b = 0; b < kMaxBC; ++b) {
        d.bc_kind[b] = b < p.n_bc ? p.bc[b].kind : BC_OUTFLOW;
        d.bc_rho[b] = p.bc[b].rho;
        d.bc_u[b] = p.bc[b].u;
        d.bc_v[b] = p.bc[b].v;
        d.bc_p[b] = p.bc[b].p;
        d.bc_Tw[b] = p.bc[b].Tw;
    }
    d.rho_min = p.min_density;
    d.rho_max = p.max_density;
    d.density_constrained = p.density_constrained;
    d.dt_mode = p.dt_mode;
    d.visc_model = p.viscosity;
    d.art_visc = p.art_viscosity;
    d.limiter = p.limiter;
    return d;
}

template <class T>
cudaError_t upload(T *dst, const std::vector<T> &src) {
    if (src.empty()) return cudaSuccess;
    return cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
}

}  // namespace

extern "C" {

int gd2d_abi_version(void) { return GD2D_ABI_VERSION; }

const char *gd2d_last_error(const gd2d_handle *h) { return h ? h->err.c_str() : g_setup_error.c_str(); }

}  // extern "C"

// Error message of handle-less entry points, read back by gd2d_last_error(NULL).
void gd2d::set_handleless_error(const char *msg) { g_setup_error = msg; }

extern "C" {

int gd2d_setup(gd2d_handle **out, int32_t n_cases, const gd2d_mesh_view *meshes, const gd2d_params *params,
               const gd2d_launch *launch) {
    if (!out) return fail(nullptr, GD2D_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (n_cases < 1 || !meshes || !params) return fail(nullptr, GD2D_ERR_ARG, "need n_cases >= 1, meshes, params");
    for (int c = 0; c < n_cases; ++c) {
        const gd2d_params &p = params[c];
        if (p.n_bc < 0 || p.n_bc > GD2D_MAX_BC) return fail(nullptr, GD2D_ERR_ARG, "case %d: n_bc out of range", c);
        if (p.flux != params[0].flux || p.viscosity != params[0].viscosity ||
            (p.viscosity != GD2D_VISC_NONE) != (params[0].viscosity != GD2D_VISC_NONE))
            return fail(nullptr, GD2D_ERR_ARG, "flux and viscosity model must agree across the cases of a handle");
        if (p.flux < 1 || p.flux > 3) return fail(nullptr, GD2D_ERR_ARG, "case %d: unknown flux %d", c, p.flux);
        if (p.limiter < 0 || p.limiter > 4) return fail(nullptr, GD2D_ERR_ARG, "case %d: unknown limiter", c);
        if (p.viscosity < 0 || p.viscosity > 3) return fail(nullptr, GD2D_ERR_ARG, "case %d: unknown viscosity", c);
        if (p.dt_mode < 0 || p.dt_mode > 2) return fail(nullptr, GD2D_ERR_ARG, "case %d: unknown dt_mode", c);
        if (!(p.Gamma > 1.0) || !(p.RGAS > 0.0)) return fail(nullptr, GD2D_ERR_ARG, "case %d: bad thermo", c);
        if (p.dt_mode == GD2D_DT_FIXED && !(p.dt > 0.0)) return fail(nullptr, GD2D_ERR_ARG, "case %d: dt <= 0", c);
        if (p.dt_mode != GD2D_DT_FIXED && !(p.CFL > 0.0)) return fail(nullptr, GD2D_ERR_ARG, "case %d: CFL <= 0", c);
        if (p.viscosity == GD2D_VISC_SUTHERLAND && !(p.T_ref > 0.0 && p.Pr > 0.0))
            return fail(nullptr, GD2D_ERR_ARG, "case %d: Sutherland needs T_ref > 0 and Pr > 0", c);
        if (p.viscosity == GD2D_VISC_CONSTANT && !(p.Pr > 0.0))
            return fail(nullptr, GD2D_ERR_ARG, "case %d: needs Pr > 0", c);
        for (int b = 0; b < p.n_bc; ++b) {
            if (p.bc[b].tag >= 0) return fail(nullptr, GD2D_ERR_ARG, "case %d: bc tags must be negative", c);
            if (p.bc[b].kind < 1 || p.bc[b].kind > 5) return fail(nullptr, GD2D_ERR_ARG, "case %d: bad bc kind", c);
            if (p.bc[b].kind == GD2D_BC_NOSLIP_ISOTHERMAL && !(p.bc[b].Tw > 0.0))
                return fail(nullptr, GD2D_ERR_ARG, "case %d: isothermal wall needs Tw > 0", c);
        }
        int rc = validate_mesh(c, meshes[c], p);
        if (rc != GD2D_OK) return rc;
    }

    gd2d_handle *h = new gd2d_handle();
    h->ncases = n_cases;
    if (launch) h->launch = *launch;
    if (h->launch.precision != GD2D_PREC_F64 && h->launch.precision != GD2D_PREC_MIXED) {
        delete h;
        return fail(nullptr, GD2D_ERR_ARG, "unknown precision %d", launch->precision);
    }
    h->mixed = h->launch.precision == GD2D_PREC_MIXED;
    int block = h->launch.block ? h->launch.block : 256;
    if (block != 128 && block != 256) {
        delete h;
        return fail(nullptr, GD2D_ERR_ARG, "block must be 128 or 256");
    }
    h->lc.block = block;
    // node-side passes: 64-thread blocks measured fastest (finer-grained
    // scheduling of their gathers; 2% of the step on the 2.09M-cell cylinder)
    h->lc.node_block = h->launch.node_block ? h->launch.node_block : 64;
    if (h->lc.node_block != 64 && h->lc.node_block != 128 && h->lc.node_block != 256) {
        delete h;
        return fail(nullptr, GD2D_ERR_ARG, "node_block must be 64, 128 or 256");
    }
    h->lc.persistent = h->launch.persistent;
    // register budget of the cell kernel, measured best on the 2.09M-cell
    // viscous cylinder: 3 blocks/SM for the FP64 kernels (the tile-face
    // kernel holds its next face record through the current face), 4 for
    // the mixed kernels
    h->lc.min_blocks = h->launch.min_blocks ? h->launch.min_blocks : (h->mixed ? 4 : 3);
    if (h->lc.min_blocks < 2 || h->lc.min_blocks > 4) {
        delete h;
        return fail(nullptr, GD2D_ERR_ARG, "min_blocks must be 2, 3 or 4");
    }
    h->loop = h->launch.loop;
    if (h->loop < GD2D_LOOP_CELL || h->loop > GD2D_LOOP_TILE_FACES) {
        delete h;
        return fail(nullptr, GD2D_ERR_ARG, "unknown loop variant %d", h->loop);
    }
    if (h->loop != GD2D_LOOP_CELL && h->loop != GD2D_LOOP_TILE_FACES && h->mixed) {
        delete h;
        return fail(nullptr, GD2D_ERR_ARG, "the face-loop variants run the FP64 path only");
    }
    h->graph_steps = h->launch.graph_steps > 0 ? h->launch.graph_steps : 32;
    h->flux = params[0].flux;
    h->visc = params[0].viscosity != GD2D_VISC_NONE;
    {
        // the library links its own CUDA runtime: the caller's current
        // device does not carry over, the launch record names the device
        int ndev = 0;
        cudaError_t e = cudaGetDeviceCount(&ndev);
        if (e != cudaSuccess) {
            delete h;
            return fail(nullptr, GD2D_ERR_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
        }
        if (h->launch.device < 0 || h->launch.device >= ndev) {
            delete h;
            return fail(nullptr, GD2D_ERR_ARG, "device %d out of range (%d devices)", h->launch.device, ndev);
        }
        h->device = h->launch.device;
        e = cudaSetDevice(h->device);
        if (e != cudaSuccess) {
            delete h;
            return fail(nullptr, GD2D_ERR_CUDA, "cudaSetDevice(%d): %s", h->device, cudaGetErrorString(e));
        }
    }
    if (h->launch.stream) {
        h->stream = (cudaStream_t)h->launch.stream;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete h;
            return fail(nullptr, GD2D_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
        }
        h->own_stream = true;
    }

    // ------------------------------------------------------- ordering
    h->cases.resize(n_cases);
    int64_t Nc = 0, Nn = 0, NcRef = 0, NnRef = 0;
    int W = 1;
    bool unit = true;
    for (int c = 0; c < n_cases; ++c) {
        const gd2d_mesh_view &mv = meshes[c];
        HostCase &hc = h->cases[c];
        hc.nc = mv.n_cells;
        hc.nn = mv.n_nodes;
        hc.params = params[c];
        hc.start_time = params[c].start_time;
        hc.nc_pad = (hc.nc + kCellPad - 1) / kCellPad * kCellPad;
        hc.cell_off = Nc;
        hc.node_off = Nn;
        hc.ref_off = NcRef;
        hc.nref_off = NnRef;
        NcRef += hc.nc;
        NnRef += hc.nn;
        Nc += hc.nc_pad;
        Nn += (hc.nn + 3) / 4 * 4;
        for (int b = 0; b < params[c].n_bc; ++b) h->tgv |= params[c].bc[b].kind == GD2D_BC_TGV_ANALYTIC;
        for (int64_t i = 0; i < hc.nc; ++i) h->quads |= mv.mesh_connectivity[cidx(hc.nc, i, 2)] == 4;
        const int order = h->launch.order;
        if (order == GD2D_ORDER_HILBERT) {
            std::vector<double> xs(hc.nc), ys(hc.nc);
            for (int64_t i = 0; i < hc.nc; ++i) {
                xs[i] = mv.cell_mid_points[cidx(hc.nc, i, 0)];
                ys[i] = mv.cell_mid_points[cidx(hc.nc, i, 1)];
            }
            hilbert_order(xs, ys, hc.cell_perm);
            std::vector<double> nx(mv.x_nodes, mv.x_nodes + hc.nn), ny(mv.y_nodes, mv.y_nodes + hc.nn);
            hilbert_order(nx, ny, hc.node_perm);
        } else if (order == GD2D_ORDER_RCM) {
            rcm_order(mv, hc.cell_perm);
            hc.node_perm.resize(hc.nn);
            std::iota(hc.node_perm.begin(), hc.node_perm.end(), 0);
        } else {
            hc.cell_perm.resize(hc.nc);
            std::iota(hc.cell_perm.begin(), hc.cell_perm.end(), 0);
            hc.node_perm.resize(hc.nn);
            std::iota(hc.node_perm.begin(), hc.node_perm.end(), 0);
        }
        if (order == GD2D_ORDER_RCM) {
            // nodes in order of first use by the reordered cells
            std::vector<char> seen(hc.nn, 0);
            std::vector<int64_t> np;
            np.reserve(hc.nn);
            for (int64_t j = 0; j < hc.nc; ++j) {
                int64_t i = hc.cell_perm[j];
                int nf = mv.mesh_connectivity[cidx(hc.nc, i, 2)];
                for (int q = 0; q < nf; ++q) {
                    int32_t v = mv.mesh_connectivity[cidx(hc.nc, i, 3 + q)] - 1;
                    if (v >= 0 && v < hc.nn && !seen[v]) { seen[v] = 1; np.push_back(v); }
                }
            }
            for (int64_t v = 0; v < hc.nn; ++v) if (!seen[v]) np.push_back(v);
            hc.node_perm.swap(np);
        }
        hc.cell_inv.assign(hc.nc, 0);
        for (int64_t j = 0; j < hc.nc; ++j) hc.cell_inv[hc.cell_perm[j]] = j;
        hc.node_inv.assign(hc.nn, 0);
        for (int64_t j = 0; j < hc.nn; ++j) hc.node_inv[hc.node_perm[j]] = j;
        for (int64_t J = 0; J < hc.nn; ++J) {
            int cnt = 0;
            for (int j = 0; j < mv.n_neib_cells; ++j) {
                int32_t cc = mv.cell_clusters[cidx(hc.nn, J, j)];
                if (cc != 0) {
                    ++cnt;
                    if (mv.node_stencils[cidx(hc.nn, J, j)] != 1.0) unit = false;
                }
            }
            W = std::max(W, cnt);
        }
    }
    const int nfmax = h->quads ? 4 : 3;
    const int64_t ntiles = Nc / block;

    // ------------------------------------------------------- packing
    std::vector<int4> nbr(Nc), dn(Nc), up(Nc), dn2, up2;
    std::vector<int2> c2n((size_t)nfmax * Nc, make_int2(0, 0));
    std::vector<double> gnx((size_t)nfmax * Nc, 0.0), gny((size_t)nfmax * Nc, 0.0), glen((size_t)nfmax * Nc, 0.0);
    std::vector<double> rarea(Nc, 0.0), area(Nc, 0.0), hx(Nc, 0.0), charlen(Nc, 0.0);
    std::vector<double2> mid;
    std::vector<double> xnode, ynode;
    std::vector<int32_t> cl((size_t)W * Nn, -1);
    std::vector<double> wt;
    if (!unit) wt.assign((size_t)W * Nn, 0.0);
    if (h->quads) { dn2.assign(Nc, make_int4(0, 0, 0, 0)); up2.assign(Nc, make_int4(0, 0, 0, 0)); }
    if (h->tgv) { mid.assign(Nc, make_double2(0.0, 0.0)); xnode.assign(Nn, 0.0); ynode.assign(Nn, 0.0); }
    for (int64_t g = 0; g < Nc; ++g) nbr[g] = make_int4(kAbsent, kAbsent, kAbsent, kAbsent);
    for (int64_t g = 0; g < Nc; ++g) { dn[g] = make_int4(0, 0, 0, 0); up[g] = make_int4(0, 0, 0, 0); }
    std::vector<int32_t> tile_case(ntiles, 0);
    std::vector<int32_t> node_case(Nn, 0);
    h->hcases.resize(n_cases);
    int64_t ngroups = 0;
    for (int c = 0; c < n_cases; ++c) {
        const gd2d_mesh_view &mv = meshes[c];
        HostCase &hc = h->cases[c];
        const int64_t n = hc.nc, nn = hc.nn;
        double maxEdge = mv.HX[0];
        for (int64_t i = 1; i < n; ++i) maxEdge = std::max(maxEdge, mv.HX[i]);
        auto node_g = [&](int32_t id1) -> int32_t {  // 1-based reference id -> global new id
            if (id1 < 1) return 0;
            return (int32_t)(hc.node_off + hc.node_inv[id1 - 1]);
        };
        for (int64_t j = 0; j < n; ++j) {
            const int64_t i = hc.cell_perm[j];
            const int64_t g = hc.cell_off + j;
            const int nf = mv.mesh_connectivity[cidx(n, i, 2)];
            int nb[4] = {kAbsent, kAbsent, kAbsent, kAbsent};
            int d1[4] = {0, 0, 0, 0}, u1[4] = {0, 0, 0, 0}, d2[4] = {0, 0, 0, 0}, u2[4] = {0, 0, 0, 0};
            double per = 0.0;
            for (int k = 0; k < nf; ++k) {
                int32_t st = mv.cell_stiffness[cidx(n, i, k)];
                if (st >= 1) {
                    nb[k] = (int32_t)(hc.cell_off + hc.cell_inv[st - 1]);
                    d1[k] = node_g(mv.node2cellL2down[cidx(n, i, 2 * k)]);
                    u1[k] = node_g(mv.node2cellL2up[cidx(n, i, 2 * k)]);
                    if (nf == 4) {
                        d2[k] = node_g(mv.node2cellL2down[cidx(n, i, 2 * k + 1)]);
                        u2[k] = node_g(mv.node2cellL2up[cidx(n, i, 2 * k + 1)]);
                    }
                } else {
                    int slot = 0;
                    for (int b = 0; b < hc.params.n_bc; ++b) if (hc.params.bc[b].tag == st) { slot = b; break; }
                    nb[k] = -(slot + 1);
                }
                const size_t o = (size_t)k * Nc + g;
                gnx[o] = mv.cell_edges_Nx[cidx(n, i, k)];
                gny[o] = mv.cell_edges_Ny[cidx(n, i, k)];
                glen[o] = mv.cell_edges_length[cidx(n, i, k)];
                c2n[o] = make_int2(node_g(mv.cells2nodes[cidx(n, i, 2 * k)]), node_g(mv.cells2nodes[cidx(n, i, 2 * k + 1)]));
                per += mv.cell_edges_length[cidx(n, i, k)];
            }
            nbr[g] = make_int4(nb[0], nb[1], nb[2], nb[3]);
            dn[g] = make_int4(d1[0], d1[1], d1[2], d1[3]);
            up[g] = make_int4(u1[0], u1[1], u1[2], u1[3]);
            if (h->quads) { dn2[g] = make_int4(d2[0], d2[1], d2[2], d2[3]); up2[g] = make_int4(u2[0], u2[1], u2[2], u2[3]); }
            const double A = mv.cell_areas[i];
            area[g] = A;
            rarea[g] = 1.0 / A;
            hx[g] = mv.HX[i];
            charlen[g] = 2.0 * A / per;
            if (h->tgv) mid[g] = make_double2(mv.cell_mid_points[cidx(n, i, 0)], mv.cell_mid_points[cidx(n, i, 1)]);
        }
        for (int64_t j = 0; j < nn; ++j) {
            const int64_t J = hc.node_perm[j];
            const int64_t gn = hc.node_off + j;
            int slot = 0;
            for (int q = 0; q < mv.n_neib_cells; ++q) {
                int32_t cc = mv.cell_clusters[cidx(nn, J, q)];
                if (cc != 0) {
                    cl[(size_t)slot * Nn + gn] = (int32_t)(hc.cell_off + hc.cell_inv[cc - 1]);
                    if (!unit) wt[(size_t)slot * Nn + gn] = mv.node_stencils[cidx(nn, J, q)];
                    ++slot;
                }
            }
            if (h->tgv) { xnode[gn] = mv.x_nodes[J]; ynode[gn] = mv.y_nodes[J]; }
        }
        DevCase d = make_devcase(hc.params, maxEdge);
        d.cell_begin = hc.cell_off;
        d.cell_end = hc.cell_off + hc.nc_pad;
        d.tile_begin = hc.cell_off / block;
        d.tile_end = (hc.cell_off + hc.nc_pad) / block;
        d.group_begin = ngroups;
        ngroups += (d.tile_end - d.tile_begin + kGroupTiles - 1) / kGroupTiles;
        d.group_end = ngroups;
        for (int64_t t = d.tile_begin; t < d.tile_end; ++t) tile_case[t] = c;
        const int64_t node_end = (c + 1 < n_cases) ? h->cases[c + 1].node_off : Nn;
        for (int64_t j = hc.node_off; j < node_end; ++j) node_case[j] = c;
        h->hcases[c] = d;
    }
    h->tile_case_h = tile_case;
    h->ngroups = ngroups;

    // face list for the face-loop variants: each interior face once (from its
    // lower-indexed cell), boundary faces once; greedy edge colouring so that
    // no two faces of one colour share a cell
    std::vector<int4> faces;
    auto code_k = [](const int4 &v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); };
    if (h->loop == GD2D_LOOP_FACE_COLOURED || h->loop == GD2D_LOOP_FACE_SLOTS) {
        std::vector<uint8_t> used(Nc, 0);
        std::vector<int> colour;
        for (int64_t g = 0; g < Nc; ++g) {
            const int4 nb = nbr[g];
            if (nb.x == kAbsent) continue;
            const int nf = nb.w != kAbsent ? 4 : 3;
            for (int k = 0; k < nf; ++k) {
                const int code = code_k(nb, k);
                if (code >= 0 && code < g) continue;
                int kb = 0;
                uint8_t mask = used[g];
                if (code >= 0) {
                    for (int q = 0; q < 4; ++q)
                        if (code_k(nbr[code], q) == (int)g) kb = q;
                    mask |= used[code];
                }
                int col = 0;
                while (mask & (1u << col)) ++col;
                used[g] |= (uint8_t)(1u << col);
                if (code >= 0) used[code] |= (uint8_t)(1u << col);
                faces.push_back(make_int4((int)g, code, k | (kb << 8), col));
                colour.push_back(col);
            }
        }
        std::stable_sort(faces.begin(), faces.end(), [](const int4 &a, const int4 &b) { return a.w < b.w; });
        const int ncol = faces.empty() ? 0 : faces.back().w + 1;
        h->colour_off.assign(ncol + 1, 0);
        for (const int4 &f : faces) h->colour_off[f.w + 1]++;
        for (int c = 0; c < ncol; ++c) h->colour_off[c + 1] += h->colour_off[c];
        h->nfaces = (int64_t)faces.size();
    }

    // tile-local face lists: every face slot of a tile's cells, except that a
    // face between two cells of the same tile is listed once (from the
    // lower-indexed cell, its flux stored negated into the other cell's slot)
    // when the other cell's evaluation of it is the exact negation: AUSM+
    // with the Minmod or Venkatakrishnan limiter or none (the flux, the
    // limiter and the role-aware epsilon are antisymmetric bit for bit),
    // normals exactly negated, equal lengths, down/up nodes exchanged, both
    // cells of the same kind and exactly one slot of each facing the other
    std::vector<int64_t> tf_off;
    std::vector<int4> tf_rec;
    std::vector<int2> tf_q, tf_e;
    std::vector<double> tf_nx, tf_ny, tf_len;
    if (h->loop == GD2D_LOOP_TILE_FACES) {
        std::vector<char> case_pairs(n_cases, 0);
        for (int c = 0; c < n_cases; ++c) {
            const int lim = params[c].limiter;
            case_pairs[c] = h->flux == GD2D_FLUX_AUSM_PLUS &&
                            (lim == GD2D_LIM_NONE || lim == GD2D_LIM_MINMOD || lim == GD2D_LIM_VENKAT);
        }
        auto slot_facing = [&](int64_t b, int64_t a, int *count) {
            int kb = -1;
            *count = 0;
            for (int q = 0; q < 4; ++q)
                if (code_k(nbr[b], q) == (int)a) { kb = q; ++*count; }
            return kb;
        };
        auto is_quad_cell = [&](int64_t g) { return h->quads && nbr[g].w != kAbsent; };
        // (lo, klo) and (hi, khi): the two slots of one face, lo < hi
        auto pairable = [&](int64_t lo, int klo, int64_t hi, int khi) {
            if (!case_pairs[tile_case[lo / block]]) return false;
            if (is_quad_cell(lo) != is_quad_cell(hi)) return false;
            const size_t ol = (size_t)klo * Nc + lo, oh = (size_t)khi * Nc + hi;
            if (!(gnx[oh] == -gnx[ol] && gny[oh] == -gny[ol] && glen[oh] == glen[ol])) return false;
            if (code_k(dn[hi], khi) != code_k(up[lo], klo) || code_k(up[hi], khi) != code_k(dn[lo], klo)) return false;
            if (is_quad_cell(lo) && (code_k(dn2[hi], khi) != code_k(up2[lo], klo) ||
                                     code_k(up2[hi], khi) != code_k(dn2[lo], klo)))
                return false;
            // the viscous edge terms are negated for the other cell too: the
            // two slots name the same pair of edge nodes (in either order)
            if (h->visc) {
                const int2 el = c2n[ol], eh = c2n[oh];
                if (!((el.x == eh.x && el.y == eh.y) || (el.x == eh.y && el.y == eh.x))) return false;
            }
            return true;
        };
        tf_off.assign(ntiles + 1, 0);
        for (int64_t t = 0; t < ntiles; ++t) {
            for (int la = 0; la < block; ++la) {
                const int64_t g = t * block + la;
                const int4 nb = nbr[g];
                if (nb.x == kAbsent) continue;
                const bool quad = is_quad_cell(g);
                const int nf = quad ? 4 : 3;
                for (int k = 0; k < nf; ++k) {
                    const int code = code_k(nb, k);
                    int lbp = 0, kb = 0;
                    if (code >= 0 && code != g && code / block == t) {
                        int cb = 0, ca = 0;
                        const int kk = slot_facing(code, g, &cb);
                        slot_facing(g, code, &ca);
                        if (kk >= 0 && cb == 1 && ca == 1) {
                            const bool ok = (g < code) ? pairable(g, k, code, kk) : pairable(code, kk, g, k);
                            if (ok) {
                                if (code < g) continue;  // listed by the other cell
                                lbp = (int)(code - t * block) + 1;
                                kb = kk;
                            }
                        }
                    }
                    tf_rec.push_back(make_int4(code, pack_tile_face(la, k, lbp, kb, quad), code_k(dn[g], k),
                                               code_k(up[g], k)));
                    if (h->quads) tf_q.push_back(make_int2(code_k(dn2[g], k), code_k(up2[g], k)));
                    const size_t o = (size_t)k * Nc + g;
                    if (h->visc) tf_e.push_back(c2n[o]);
                    tf_nx.push_back(gnx[o]);
                    tf_ny.push_back(gny[o]);
                    tf_len.push_back(glen[o]);
                }
            }
            tf_off[t + 1] = (int64_t)tf_rec.size();
        }
        h->nfaces = (int64_t)tf_rec.size();
        if (h->nfaces >= (int64_t)INT32_MAX) {  // the tile kernels index faces with 32 bits
            if (h->own_stream) cudaStreamDestroy(h->stream);
            delete h;
            return fail(nullptr, GD2D_ERR_ARG, "%lld tile faces: more than the tile-face loop supports",
                        (long long)tf_rec.size());
        }
    }

    // ------------------------------------------------------- device
    cudaSetDevice(h->device);
    DevMesh &m = h->m;
    DevState &s = h->s;
    m.Nc = Nc; m.Nn = Nn; m.ncases = n_cases; m.nfmax = nfmax; m.cluster_w = W; m.unit_weights = unit ? 1 : 0;
    m.ntiles = ntiles;
    int4 *d_nbr, *d_dn, *d_up, *d_dn2 = nullptr, *d_up2 = nullptr;
    int2 *d_c2n;
    double *d_nx, *d_ny, *d_len, *d_rarea, *d_area, *d_hx, *d_charlen, *d_xn = nullptr, *d_yn = nullptr, *d_wt = nullptr;
    double2 *d_mid = nullptr;
    int32_t *d_cl, *d_tc, *d_nc = nullptr;
    DevCase *d_cases;
    auto bail = [&](int rc) {
        h->buf.free_all();
        if (h->ring_host) cudaFreeHost(h->ring_host);
        if (h->h_stage) cudaFreeHost(h->h_stage);
        for (auto &e : h->ev_total) if (e) cudaEventDestroy(e);
        for (auto &e : h->ev_eager) if (e) cudaEventDestroy(e);
        if (h->own_stream) cudaStreamDestroy(h->stream);
        g_setup_error = h->err;
        delete h;
        return rc;
    };
#define ALLOC(ptr, n)                                                                              \
    do {                                                                                           \
        cudaError_t e__ = h->buf.alloc(&(ptr), (size_t)(n));                                       \
        if (e__ != cudaSuccess) return bail(fail(h, GD2D_ERR_OOM, "cudaMalloc %s: %s", #ptr, cudaGetErrorString(e__))); \
    } while (0)
#define UPLOAD(ptr, vec)                                                                           \
    do {                                                                                           \
        cudaError_t e__ = upload((ptr), (vec));                                                    \
        if (e__ != cudaSuccess) return bail(fail(h, GD2D_ERR_CUDA, "upload %s: %s", #ptr, cudaGetErrorString(e__))); \
    } while (0)
    ALLOC(d_nbr, Nc); UPLOAD(d_nbr, nbr);
    ALLOC(d_dn, Nc); UPLOAD(d_dn, dn);
    ALLOC(d_up, Nc); UPLOAD(d_up, up);
    if (h->quads) { ALLOC(d_dn2, Nc); UPLOAD(d_dn2, dn2); ALLOC(d_up2, Nc); UPLOAD(d_up2, up2); }
    ALLOC(d_c2n, (size_t)nfmax * Nc); UPLOAD(d_c2n, c2n);
    if (!h->mixed) {
        ALLOC(d_nx, (size_t)nfmax * Nc); UPLOAD(d_nx, gnx);
        ALLOC(d_ny, (size_t)nfmax * Nc); UPLOAD(d_ny, gny);
        ALLOC(d_len, (size_t)nfmax * Nc); UPLOAD(d_len, glen);
        ALLOC(d_rarea, Nc); UPLOAD(d_rarea, rarea);
        ALLOC(d_area, Nc); UPLOAD(d_area, area);
        ALLOC(d_hx, Nc); UPLOAD(d_hx, hx);
        ALLOC(d_charlen, Nc); UPLOAD(d_charlen, charlen);
    } else {
        d_nx = d_ny = d_len = d_rarea = d_area = d_hx = d_charlen = nullptr;
        auto to_f = [](const std::vector<double> &v) {
            std::vector<float> f(v.size());
            for (size_t i = 0; i < v.size(); ++i) f[i] = (float)v[i];
            return f;
        };
        float *f_nx, *f_ny, *f_len, *f_rarea, *f_area, *f_hx, *f_charlen;
        ALLOC(f_nx, (size_t)nfmax * Nc); UPLOAD(f_nx, to_f(gnx));
        ALLOC(f_ny, (size_t)nfmax * Nc); UPLOAD(f_ny, to_f(gny));
        ALLOC(f_len, (size_t)nfmax * Nc); UPLOAD(f_len, to_f(glen));
        ALLOC(f_rarea, Nc); UPLOAD(f_rarea, to_f(rarea));
        ALLOC(f_area, Nc); UPLOAD(f_area, to_f(area));
        ALLOC(f_hx, Nc); UPLOAD(f_hx, to_f(hx));
        ALLOC(f_charlen, Nc); UPLOAD(f_charlen, to_f(charlen));
        m.nxf = f_nx; m.nyf = f_ny; m.lenf = f_len; m.rareaf = f_rarea; m.areaf = f_area; m.hxf = f_hx;
        m.charlenf = f_charlen;
        if (h->visc) {
            // the first gradient's edge weights, one plane each instead of
            // three (normal components and length)
            std::vector<float> nlx((size_t)nfmax * Nc), nly((size_t)nfmax * Nc);
            for (size_t i = 0; i < nlx.size(); ++i) {
                nlx[i] = (float)(gnx[i] * glen[i]);
                nly[i] = (float)(gny[i] * glen[i]);
            }
            float *f_nlx, *f_nly;
            ALLOC(f_nlx, nlx.size()); UPLOAD(f_nlx, nlx);
            ALLOC(f_nly, nly.size()); UPLOAD(f_nly, nly);
            m.nlxf = f_nlx; m.nlyf = f_nly;
        }
    }
    if (h->tgv) {
        ALLOC(d_mid, Nc); UPLOAD(d_mid, mid);
        ALLOC(d_xn, Nn); UPLOAD(d_xn, xnode);
        ALLOC(d_yn, Nn); UPLOAD(d_yn, ynode);
    }
    ALLOC(d_cl, (size_t)W * Nn); UPLOAD(d_cl, cl);
    if (!unit) { ALLOC(d_wt, (size_t)W * Nn); UPLOAD(d_wt, wt); }
    ALLOC(d_tc, ntiles); UPLOAD(d_tc, tile_case);
    if (h->visc) { ALLOC(d_nc, Nn); UPLOAD(d_nc, node_case); }
    ALLOC(d_cases, n_cases); UPLOAD(d_cases, h->hcases);
    m.nbr = d_nbr; m.dn = d_dn; m.up = d_up; m.dn2 = d_dn2; m.up2 = d_up2; m.c2n = d_c2n;
    m.nx = d_nx; m.ny = d_ny; m.len = d_len; m.rarea = d_rarea; m.area = d_area; m.hx = d_hx; m.charlen = d_charlen;
    m.mid = d_mid; m.xnode = d_xn; m.ynode = d_yn; m.cl = d_cl; m.wt = d_wt; m.tile_case = d_tc; m.node_case = d_nc;
    m.cases = d_cases;

    s.ring_len = 1024;
    ALLOC(s.U, Nc);
    if (!h->mixed) {
        ALLOC(s.prim, 2 * Nc);
        ALLOC(s.nodeP, Nn);
        if (h->visc) { ALLOC(s.nodeC, Nn); ALLOC(s.g1, Nc); ALLOC(s.nodeG, Nn); }
    } else {
        ALLOC(s.primf, 2 * Nc);
        ALLOC(s.nodePf, Nn);
        if (h->visc) { ALLOC(s.nodeCf, Nn); ALLOC(s.g1f, Nc); ALLOC(s.nodeGf, Nn); }
    }
    ALLOC(s.part, (size_t)ntiles * kPartials);
    if (h->loop == GD2D_LOOP_TILE_FACES) {
        int64_t *d_tfo;
        int4 *d_tfr;
        int2 *d_tfq = nullptr;
        ALLOC(d_tfo, tf_off.size()); UPLOAD(d_tfo, tf_off);
        ALLOC(d_tfr, tf_rec.size()); UPLOAD(d_tfr, tf_rec);
        if (h->quads) { ALLOC(d_tfq, tf_q.size()); UPLOAD(d_tfq, tf_q); }
        if (h->visc) {
            int2 *d_tfe;
            ALLOC(d_tfe, tf_e.size()); UPLOAD(d_tfe, tf_e);
            m.tf_e = d_tfe;
        }
        if (h->mixed) {
            // (the FP64 tile kernel reads the face geometry from the per-cell
            // planes, which its viscous source reads too)
            auto to_f = [](const std::vector<double> &v) {
                std::vector<float> f(v.size());
                for (size_t i = 0; i < v.size(); ++i) f[i] = (float)v[i];
                return f;
            };
            float *f_nx, *f_ny, *f_len;
            ALLOC(f_nx, tf_nx.size()); UPLOAD(f_nx, to_f(tf_nx));
            ALLOC(f_ny, tf_ny.size()); UPLOAD(f_ny, to_f(tf_ny));
            ALLOC(f_len, tf_len.size()); UPLOAD(f_len, to_f(tf_len));
            m.tf_nxf = f_nx; m.tf_nyf = f_ny; m.tf_lenf = f_len;
        }
        m.tf_off = d_tfo; m.tf_rec = d_tfr; m.tf_q = d_tfq;
    }
    if (h->loop == GD2D_LOOP_FACE_COLOURED || h->loop == GD2D_LOOP_FACE_SLOTS) {
        ALLOC(h->d_faces, faces.size()); UPLOAD(h->d_faces, faces);
        if (h->loop == GD2D_LOOP_FACE_COLOURED) ALLOC(h->Facc, Nc);
        else ALLOC(h->Fslot, (size_t)nfmax * Nc);
    }
    ALLOC(s.cstate, n_cases);
    ALLOC(s.ring, (size_t)s.ring_len * n_cases);
    ALLOC(s.parity, 1);
    ALLOC(s.node_done, 1);
    ALLOC(s.gpart, (size_t)ngroups * kPartials);
    {
        std::vector<int32_t> group_case((size_t)ngroups, 0);
        for (int c = 0; c < n_cases; ++c)
            for (int64_t gi = h->hcases[c].group_begin; gi < h->hcases[c].group_end; ++gi) group_case[gi] = c;
        int32_t *d_gc;
        ALLOC(d_gc, group_case.size()); UPLOAD(d_gc, group_case);
        m.group_case = d_gc;
        m.ngroups = ngroups;
    }
    {
        std::vector<int32_t> perm(Nc, 0), inv(NcRef, 0), ninv(NnRef, 0);
        int64_t maxrows = 1;
        for (const HostCase &hc : h->cases) {
            for (int64_t j = 0; j < hc.nc; ++j) perm[hc.cell_off + j] = (int32_t)hc.cell_perm[j];
            for (int64_t i = 0; i < hc.nc; ++i) inv[hc.ref_off + i] = (int32_t)hc.cell_inv[i];
            for (int64_t i = 0; i < hc.nn; ++i) ninv[hc.nref_off + i] = (int32_t)hc.node_inv[i];
            maxrows = std::max(maxrows, std::max(hc.nc, hc.nn));
        }
        ALLOC(h->d_perm, perm.size()); UPLOAD(h->d_perm, perm);
        ALLOC(h->d_inv, inv.size()); UPLOAD(h->d_inv, inv);
        ALLOC(h->d_ninv, ninv.size()); UPLOAD(h->d_ninv, ninv);
        ALLOC(h->d_stage, (size_t)4 * maxrows);
        cudaError_t e = cudaMallocHost((void **)&h->h_stage, sizeof(double) * 4 * (size_t)maxrows);
        if (e != cudaSuccess) return bail(fail(h, GD2D_ERR_OOM, "cudaMallocHost: %s", cudaGetErrorString(e)));
    }
#undef ALLOC
#undef UPLOAD
    {
        int dev_sms = 148;
        cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, h->device);
        h->lc.grid = dev_sms * h->lc.min_blocks * (256 / block);
    }
    h->history.assign(n_cases, {});
    h->cs_host.assign(n_cases, CaseState{});
    cudaEventCreate(&h->ev_total[0]);
    cudaEventCreate(&h->ev_total[1]);
    cudaEventCreate(&h->ev_eager[0]);
    cudaEventCreate(&h->ev_eager[1]);
    {
        // mapped: each step's finalizing warp writes its statistics row here
        // directly, so a step needs no copy before the host can read them
        cudaError_t e = cudaHostAlloc((void **)&h->ring_host, sizeof(DevStats) * (size_t)s.ring_len * n_cases,
                                      cudaHostAllocMapped);
        if (e != cudaSuccess) return bail(fail(h, GD2D_ERR_OOM, "cudaHostAlloc: %s", cudaGetErrorString(e)));
        e = cudaHostGetDevicePointer((void **)&s.ring_host, h->ring_host, 0);
        if (e != cudaSuccess) return bail(fail(h, GD2D_ERR_CUDA, "cudaHostGetDevicePointer: %s", cudaGetErrorString(e)));
    }
    // uploads above went through the legacy stream; finish them before any
    // work is queued on the handle's stream
    {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return bail(fail(h, GD2D_ERR_CUDA, "setup: %s", cudaGetErrorString(e)));
    }
    *out = h;
    return GD2D_OK;
}

// Stream-ordered copies on the handle's stream (the handle's stream does not
// synchronise with the legacy default stream).
static int copy_sync(gd2d_handle *h, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind) {
    CUDA_TRY(h, cudaMemcpyAsync(dst, src, bytes, kind, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return GD2D_OK;
}

// Transfers between a caller's host columns and the device stage go
// through the page-locked host stage in slices of 2 MB, handed out in order
// to the handle's worker threads (StagePool, at most 8 threads with the
// caller; 16 measured no faster): uploads copy a slice into the stage and queue its DMA at once,
// so the DMA engine starts after the first slice and streams while the
// other slices are copied; downloads queue every slice's DMA first and copy
// each slice out as soon as its event completes.  The stage holds a case's
// 4 columns back to back, element v * n + i for row i of column v.
constexpr size_t kSliceElems = (size_t)1 << 18;  // 2 MB of doubles

static unsigned stage_threads() {
    const unsigned nt = std::thread::hardware_concurrency();
    return std::max(1u, std::min(nt, 8u));
}

// Elements [b0, b1) of the stage, copied from (to_stage) or to the columns.
static void stage_copy(double *stage, double *const cols[4], int64_t n, size_t b0, size_t b1, bool to_stage) {
    while (b0 < b1) {
        const size_t v = b0 / (size_t)n, i = b0 % (size_t)n;
        const size_t len = std::min(b1 - b0, (size_t)n - i);
        if (to_stage) std::memcpy(stage + b0, cols[v] + i, sizeof(double) * len);
        else std::memcpy(cols[v] + i, stage + b0, sizeof(double) * len);
        b0 += len;
    }
}

// Whether a host array of n doubles is page-locked in the current context
// (allocated or registered with CUDA), first and last element alike, so
// that the copy engine can read or write it directly.  Pageable memory is
// not an error.
static bool host_pinned(const double *p, int64_t n) {
    for (const double *q : {p, p + (n > 0 ? n - 1 : 0)}) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
            (void)cudaGetLastError();
            return false;
        }
        if (a.type != cudaMemoryTypeHost) return false;
    }
    return true;
}

// Host columns -> h_stage -> d_stage (queued on the handle's stream).
// Page-locked columns are copied to d_stage directly.
static int staged_upload(gd2d_handle *h, const double *const src[4], int64_t n) {
    if (host_pinned(src[0], n) && host_pinned(src[1], n) && host_pinned(src[2], n) && host_pinned(src[3], n)) {
        for (int v = 0; v < 4; ++v) {
            const cudaError_t e = cudaMemcpyAsync(h->d_stage + (size_t)v * n, src[v], sizeof(double) * (size_t)n,
                                                  cudaMemcpyHostToDevice, h->stream);
            if (e != cudaSuccess) return fail(h, GD2D_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
        }
        return GD2D_OK;
    }
    double *cols[4] = {const_cast<double *>(src[0]), const_cast<double *>(src[1]), const_cast<double *>(src[2]),
                       const_cast<double *>(src[3])};
    const size_t total = 4 * (size_t)n;
    const unsigned ns = (unsigned)((total + kSliceElems - 1) / kSliceElems);
    std::vector<cudaError_t> err(ns, cudaSuccess);
    h->pool.run(h->device, stage_threads() - 1, ns, [&](unsigned k) {
        const size_t b0 = (size_t)k * kSliceElems, b1 = std::min(total, b0 + kSliceElems);
        stage_copy(h->h_stage, cols, n, b0, b1, true);
        err[k] = cudaMemcpyAsync(h->d_stage + b0, h->h_stage + b0, sizeof(double) * (b1 - b0),
                                 cudaMemcpyHostToDevice, h->stream);
    });
    for (cudaError_t e : err)
        if (e != cudaSuccess) return fail(h, GD2D_ERR_CUDA, "staged upload: %s", cudaGetErrorString(e));
    return GD2D_OK;
}

// d_stage -> h_stage -> a column-major (n, 4) host matrix; returns when the
// matrix is complete.  A page-locked matrix is copied to directly.
static int staged_download(gd2d_handle *h, double *dst, int64_t n) {
    const size_t total = 4 * (size_t)n;
    if (host_pinned(dst, (int64_t)total)) {
        cudaError_t e = cudaMemcpyAsync(dst, h->d_stage, sizeof(double) * total, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) {
            cudaStreamSynchronize(h->stream);
            return fail(h, GD2D_ERR_CUDA, "download: %s", cudaGetErrorString(e));
        }
        return GD2D_OK;
    }
    double *cols[4] = {dst, dst + n, dst + 2 * n, dst + 3 * n};
    const unsigned ns = (unsigned)((total + kSliceElems - 1) / kSliceElems);
    cudaError_t e = cudaSuccess;
    while (e == cudaSuccess && h->slice_ev.size() < ns) {
        cudaEvent_t x = nullptr;
        e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
        if (e == cudaSuccess) h->slice_ev.push_back(x);
    }
    for (unsigned k = 0; k < ns && e == cudaSuccess; ++k) {
        const size_t b0 = (size_t)k * kSliceElems, b1 = std::min(total, b0 + kSliceElems);
        e = cudaMemcpyAsync(h->h_stage + b0, h->d_stage + b0, sizeof(double) * (b1 - b0), cudaMemcpyDeviceToHost,
                            h->stream);
        if (e == cudaSuccess) e = cudaEventRecord(h->slice_ev[k], h->stream);
    }
    if (e != cudaSuccess) {
        cudaStreamSynchronize(h->stream);  // nothing queued above may outlive the call
        return fail(h, GD2D_ERR_CUDA, "staged download: %s", cudaGetErrorString(e));
    }
    std::vector<cudaError_t> err(ns, cudaSuccess);
    h->pool.run(h->device, stage_threads() - 1, ns, [&](unsigned k) {
        const size_t b0 = (size_t)k * kSliceElems, b1 = std::min(total, b0 + kSliceElems);
        err[k] = cudaEventSynchronize(h->slice_ev[k]);
        if (err[k] == cudaSuccess) stage_copy(h->h_stage, cols, n, b0, b1, false);
    });
    for (cudaError_t x : err)
        if (x != cudaSuccess) return fail(h, GD2D_ERR_CUDA, "staged download: %s", cudaGetErrorString(x));
    return GD2D_OK;
}

static int ensure_case(gd2d_handle *h, int32_t icase) {
    if (!h) return fail(nullptr, GD2D_ERR_ARG, "NULL handle");
    if (icase < 0 || icase >= h->ncases) return fail(h, GD2D_ERR_ARG, "case index %d out of range", icase);
    return GD2D_OK;
}

static int drop_graph(gd2d_handle *h) {
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
    if (h->graph1) { cudaGraphExecDestroy(h->graph1); h->graph1 = nullptr; }
    for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
    h->ev.clear();
    return GD2D_OK;
}

// Where the primitives of a case are written before its initialisation:
// FP64, the current primitive buffer; mixed, U, which the init kernel turns
// into conservatives while writing the FP32 primitives.
static int case_prims_dst(gd2d_handle *h, int32_t icase, double4 **dst) {
    const HostCase &hc = h->cases[icase];
    int par = 0;
    int rc = copy_sync(h, &par, h->s.parity, sizeof(int), cudaMemcpyDeviceToHost);
    if (rc) return rc;
    *dst = h->mixed ? h->s.U + hc.cell_off : h->s.prim + (int64_t)par * h->m.Nc + hc.cell_off;
    return GD2D_OK;
}

// The case's primitives, already in place (case_prims_dst), become its
// state: U, the node fields and the first dt.  With `exact_cons` (reference
// order columns on the device) U is then overwritten by those conservatives,
// before the node pass, so that a restart continues bit for bit (the
// round trip conservatives -> primitives -> conservatives is inexact).
static int init_case(gd2d_handle *h, int32_t icase, double t0, bool nodes_from_cells,
                     const double *exact_cons = nullptr) {
    HostCase &hc = h->cases[icase];
    CaseState &cs = h->cs_host[icase];
    cs = CaseState{};
    cs.t = t0;
    CUDA_TRY(h, cudaMemcpyAsync(h->s.cstate + icase, &cs, sizeof cs, cudaMemcpyHostToDevice, h->stream));
    // per-case init restricted to this case's tiles and nodes
    const DevCase &d = h->hcases[icase];
    if (h->mixed) {
        CUDA_TRY(h, launch_init_state_mixed(h->m, h->s, d.tile_begin, d.tile_end, h->lc, h->stream));
        if (exact_cons)
            CUDA_TRY(h, launch_cols_to_dev(exact_cons, h->d_perm + hc.cell_off, hc.nc, h->s.U + hc.cell_off, h->stream));
        CUDA_TRY(h, launch_node_avg_mixed(h->m, h->s, h->visc, false, !nodes_from_cells, hc.node_off,
                                          hc.node_off + hc.nn, d.group_begin, d.group_end, true, h->lc,
                                          h->stream));
    } else {
        CUDA_TRY(h, launch_init_state_f64(h->m, h->s, d.tile_begin, d.tile_end, h->lc, h->stream));
        if (exact_cons)
            CUDA_TRY(h, launch_cols_to_dev(exact_cons, h->d_perm + hc.cell_off, hc.nc, h->s.U + hc.cell_off, h->stream));
        CUDA_TRY(h, launch_node_avg_f64(h->m, h->s, h->visc, false, !nodes_from_cells, hc.node_off,
                                        hc.node_off + hc.nn, d.group_begin, d.group_end, true, h->lc,
                                        h->stream));
    }
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    hc.state_set = true;
    h->history[icase].clear();
    bool all = true;
    for (auto &c : h->cases) all &= c.state_set;
    h->state_ready = all;
    return GD2D_OK;
}

int gd2d_set_state(gd2d_handle *h, int32_t icase, const double *density, const double *ux, const double *uy,
                   const double *pressure) {
    int rc = ensure_case(h, icase);
    if (rc) return rc;
    if (!density || !ux || !uy || !pressure) return fail(h, GD2D_ERR_ARG, "NULL field pointer");
    cudaSetDevice(h->device);
    const HostCase &hc = h->cases[icase];
    double4 *dst = nullptr;
    if ((rc = case_prims_dst(h, icase, &dst))) return rc;
    const int64_t n = hc.nc;
    const double *cols[4] = {density, ux, uy, pressure};
    if ((rc = staged_upload(h, cols, n))) return rc;
    CUDA_TRY(h, launch_cols_to_dev(h->d_stage, h->d_perm + hc.cell_off, n, dst, h->stream));
    return init_case(h, icase, hc.start_time, hc.params.init_nodes != 0);
}

int gd2d_set_conservative(gd2d_handle *h, int32_t icase, const double *ucons, double flow_time, int32_t rebuild_nodes) {
    int rc = ensure_case(h, icase);
    if (rc) return rc;
    if (!ucons) return fail(h, GD2D_ERR_ARG, "NULL ucons");
    cudaSetDevice(h->device);
    const HostCase &hc = h->cases[icase];
    double4 *dst = nullptr;
    if ((rc = case_prims_dst(h, icase, &dst))) return rc;
    const int64_t n = hc.nc;
    const double *cols[4] = {ucons, ucons + n, ucons + 2 * n, ucons + 3 * n};
    if ((rc = staged_upload(h, cols, n))) return rc;
    CUDA_TRY(h, launch_cons_to_prims(h->d_stage, h->d_perm + hc.cell_off, n, hc.params.Gamma, dst, h->stream));
    return init_case(h, icase, flow_time, rebuild_nodes != 0, h->d_stage);
}

static int64_t kernels_per_step(const gd2d_handle *h) {
    // viscous gradient passes, node pass (with the group reduction)
    int64_t n = (h->visc ? 2 : 0) + 1;
    if (h->loop == GD2D_LOOP_FACE_COLOURED) n += (int64_t)h->colour_off.size() - 1 + 1;
    else if (h->loop == GD2D_LOOP_FACE_SLOTS) n += 2;
    else n += 1;
    return n;
}

// The kernels of one step on the handle's stream: [viscous gradient passes]
// -> fused cell kernel (bracketed by the optional timing events) -> node pass.
// Timing events inside a stream capture become external event-record nodes;
// outside a capture they are plain records.
static void record_timing(gd2d_handle *h, cudaEvent_t ev, bool in_capture) {
    if (in_capture) cudaEventRecordWithFlags(ev, h->stream, cudaEventRecordExternal);
    else cudaEventRecord(ev, h->stream);
}

static cudaError_t launch_step_kernels(gd2d_handle *h, cudaEvent_t before_cell, cudaEvent_t after_cell,
                                       bool in_capture = false) {
    cudaError_t e = cudaSuccess;
    if (h->visc) {
        e = h->mixed ? launch_visc_grad_mixed(h->m, h->s, h->lc, h->stream)
                     : launch_visc_grad_f64(h->m, h->s, h->lc, h->stream);
        if (e != cudaSuccess) return e;
    }
    if (before_cell) record_timing(h, before_cell, in_capture);
    if (h->loop == GD2D_LOOP_FACE_COLOURED) {
        for (size_t c = 0; c + 1 < h->colour_off.size(); ++c) {
            e = launch_face_flux_f64(h->m, h->s, h->flux, h->quads, false, h->d_faces, h->colour_off[c],
                                     h->colour_off[c + 1], h->Facc, nullptr, h->lc, h->stream);
            if (e != cudaSuccess) return e;
        }
        e = launch_face_update_f64(h->m, h->s, h->visc, h->quads, false, h->Facc, nullptr, h->lc, h->stream);
    } else if (h->loop == GD2D_LOOP_TILE_FACES) {
        e = h->mixed ? launch_cell_step_tf_mixed(h->m, h->s, h->flux, h->visc, h->quads, h->lc, h->stream)
                     : launch_cell_step_tf_f64(h->m, h->s, h->flux, h->visc, h->quads, h->lc, h->stream);
    } else if (h->loop == GD2D_LOOP_FACE_SLOTS) {
        e = launch_face_flux_f64(h->m, h->s, h->flux, h->quads, true, h->d_faces, 0, h->nfaces, nullptr, h->Fslot,
                                 h->lc, h->stream);
        if (e != cudaSuccess) return e;
        e = launch_face_update_f64(h->m, h->s, h->visc, h->quads, true, nullptr, h->Fslot, h->lc, h->stream);
    } else {
        e = h->mixed ? launch_cell_step_mixed(h->m, h->s, h->flux, h->visc, h->quads, h->lc, h->stream)
                     : launch_cell_step_f64(h->m, h->s, h->flux, h->visc, h->quads, h->lc, h->stream);
    }
    if (e != cudaSuccess) return e;
    if (after_cell) record_timing(h, after_cell, in_capture);
    // the node pass; its first blocks complete the step reduction of the
    // cell kernel's tile records
    return h->mixed ? launch_node_avg_mixed(h->m, h->s, h->visc, true, false, 0, h->m.Nn, 0, h->ngroups, false,
                                            h->lc, h->stream)
                    : launch_node_avg_f64(h->m, h->s, h->visc, true, false, 0, h->m.Nn, 0, h->ngroups, false,
                                          h->lc, h->stream);
}

// Ends the capture opened on the handle's stream in every case (a stream
// left capturing would refuse all later work) and instantiates the graph.
// A launch that failed during the capture is reported by its own error,
// which names the cause, rather than by the capture's generic invalidation;
// the partial graph is destroyed either way.
static int end_capture(gd2d_handle *h, cudaError_t launch_err, cudaGraphExec_t *out, const char *what) {
    cudaGraph_t g = nullptr;
    const cudaError_t end_err = cudaStreamEndCapture(h->stream, &g);
    if (launch_err != cudaSuccess || end_err != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        (void)cudaGetLastError();
        const cudaError_t e = launch_err != cudaSuccess ? launch_err : end_err;
        return fail(h, GD2D_ERR_CUDA, "%s: %s during %s", what, cudaGetErrorString(e),
                    launch_err != cudaSuccess ? "a kernel launch of the capture" : "cudaStreamEndCapture");
    }
    const cudaError_t e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        *out = nullptr;
        return fail(h, GD2D_ERR_CUDA, "%s: cudaGraphInstantiate: %s", what, cudaGetErrorString(e));
    }
    return GD2D_OK;
}

static int capture_graph(gd2d_handle *h, int steps, bool timing) {
    drop_graph(h);
    if (timing) {
        h->ev.resize(2 * steps);
        for (auto &e : h->ev) CUDA_TRY(h, cudaEventCreate(&e));
    }
    CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t first = cudaSuccess;
    for (int k = 0; k < steps && first == cudaSuccess; ++k) {
        first = launch_step_kernels(h, timing ? h->ev[2 * k] : nullptr, timing ? h->ev[2 * k + 1] : nullptr, true);
    }
    return end_capture(h, first, &h->graph, "step graph");
}

// A one-step graph (the remainder steps of a propagate call, and single-step
// calls), timing its cell kernel with the eager event pair.
static int capture_step_graph(gd2d_handle *h) {
    CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t first = launch_step_kernels(h, h->ev_eager[0], h->ev_eager[1], true);
    return end_capture(h, first, &h->graph1, "one-step graph");
}

int gd2d_propagate(gd2d_handle *h, int32_t nsteps, gd2d_stats *stats_out) {
    if (!h) return fail(nullptr, GD2D_ERR_ARG, "NULL handle");
    if (nsteps < 0) return fail(h, GD2D_ERR_ARG, "nsteps < 0");
    if (!h->state_ready) return fail(h, GD2D_ERR_STATE, "gd2d_set_state must be called for every case first");
    cudaSetDevice(h->device);
    const int G = h->graph_steps;
    const bool timing = true;
    int64_t launches = 0;
    double total_ms = 0.0, cell_ms = 0.0;
    int cell_samples = 0;
    int32_t done = 0;
    const int64_t RL = h->s.ring_len;
    while (done < nsteps) {
        const int32_t chunk = std::min<int32_t>(nsteps - done, h->s.ring_len);
        // steps taken so far per case, kept on the host (the device's copy
        // advances in step with it): no read-back before the launches
        std::vector<int64_t> step0(h->ncases);
        for (int c = 0; c < h->ncases; ++c) step0[c] = h->cs_host[c].step;
        // graphs this chunk needs, captured before the timed window opens
        if (G > 1 && chunk >= G && !h->graph) {
            int rc = capture_graph(h, G, timing);
            if (rc) return rc;
        }
        if (G > 1 && chunk % G != 0 && !h->graph1) {
            int rc = capture_step_graph(h);
            if (rc) return rc;
        }
        CUDA_TRY(h, cudaEventRecord(h->ev_total[0], h->stream));
        int32_t k = 0;
        bool used_graph = false;
        if (G > 1) {
            while (chunk - k >= G) {
                CUDA_TRY(h, cudaGraphLaunch(h->graph, h->stream));
                used_graph = true;
                k += G;
                launches += (int64_t)G * kernels_per_step(h);
            }
        }
        const bool time_eager = !used_graph && k < chunk;
        for (; k < chunk; ++k) {
            if (G > 1) {
                CUDA_TRY(h, cudaGraphLaunch(h->graph1, h->stream));
            } else {
                const bool last = time_eager && k == chunk - 1;
                CUDA_TRY(h, launch_step_kernels(h, last ? h->ev_eager[0] : nullptr, last ? h->ev_eager[1] : nullptr));
            }
            launches += kernels_per_step(h);
        }
        CUDA_TRY(h, cudaEventRecord(h->ev_total[1], h->stream));
        // the chunk's statistics rows are in the mapped ring once the stream
        // is idle (rows are [ring_len][ncases] and wrap; every case steps in
        // every launch, so each case's rows of this chunk are fresh)
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev_total[0], h->ev_total[1]);
        total_ms += ms;
        if (used_graph && timing && !h->ev.empty()) {
            for (int q = 0; q < G; ++q) {
                float c = 0.f;
                if (cudaEventElapsedTime(&c, h->ev[2 * q], h->ev[2 * q + 1]) == cudaSuccess) {
                    cell_ms += c;
                    ++cell_samples;
                }
            }
            (void)cudaGetLastError();  // a failed timing query must not surface at the next launch
        } else if (time_eager) {
            float c = 0.f;
            if (cudaEventElapsedTime(&c, h->ev_eager[0], h->ev_eager[1]) == cudaSuccess) {
                cell_ms += c;
                ++cell_samples;
            }
            (void)cudaGetLastError();
        }
        bool bad = false;
        for (int c = 0; c < h->ncases; ++c) {
            for (int32_t q = 0; q < chunk; ++q) {
                int64_t stp = step0[c] + q;
                const DevStats &ds = h->ring_host[(size_t)(stp % RL) * h->ncases + c];
                gd2d_stats st;
                static_assert(sizeof(gd2d_stats) == sizeof(DevStats), "stats layout");
                std::memcpy(&st, &ds, sizeof st);
                h->history[c].push_back(st);
                bad |= st.nonfinite != 0;
            }
            if (stats_out) stats_out[c] = h->history[c].back();
            h->cs_host[c].step = step0[c] + chunk;
        }
        done += chunk;
        if (bad) return fail(h, GD2D_ERR_NONFINITE, "non-finite or non-positive state after step %lld",
                             (long long)(step0[0] + chunk));
    }
    h->last_total_ms = total_ms;
    h->last_cell_ms = cell_samples ? cell_ms / cell_samples : 0.0;
    h->last_launches = launches;
    return GD2D_OK;
}

int gd2d_get_history(gd2d_handle *h, int32_t icase, gd2d_stats *out, int32_t capacity) {
    int rc = ensure_case(h, icase);
    if (rc) return rc;
    const auto &v = h->history[icase];
    int32_t n = (int32_t)std::min<size_t>(v.size(), (size_t)std::max(capacity, 0));
    if (out) std::memcpy(out, v.data() + (v.size() - n), sizeof(gd2d_stats) * n);
    return n;
}

// One device-order field of a case, reordered on the device into the
// staging columns and copied to a column-major host matrix.
static int download_rows(gd2d_handle *h, const double4 *src, const float4 *srcf, const int32_t *inv, int64_t n,
                         double *dst) {
    if (!dst) return GD2D_OK;
    CUDA_TRY(h, srcf ? launch_dev_to_cols_f(srcf, inv, n, h->d_stage, h->stream)
                     : launch_dev_to_cols(src, inv, n, h->d_stage, h->stream));
    return staged_download(h, dst, n);
}

int gd2d_get_state(gd2d_handle *h, int32_t icase, double *ucons, double *prims, double *node_prims) {
    int rc = ensure_case(h, icase);
    if (rc) return rc;
    cudaSetDevice(h->device);
    HostCase &hc = h->cases[icase];
    int par = 0;
    rc = copy_sync(h, &par, h->s.parity, sizeof(int), cudaMemcpyDeviceToHost);
    if (rc) return rc;
    const int32_t *inv = h->d_inv + hc.ref_off, *ninv = h->d_ninv + hc.nref_off;
    if ((rc = download_rows(h, h->s.U + hc.cell_off, nullptr, inv, hc.nc, ucons))) return rc;
    if (h->mixed) {
        if ((rc = download_rows(h, nullptr, h->s.primf + (int64_t)par * h->m.Nc + hc.cell_off, inv, hc.nc, prims)))
            return rc;
        if ((rc = download_rows(h, nullptr, h->s.nodePf + hc.node_off, ninv, hc.nn, node_prims))) return rc;
    } else {
        if ((rc = download_rows(h, h->s.prim + (int64_t)par * h->m.Nc + hc.cell_off, nullptr, inv, hc.nc, prims)))
            return rc;
        if ((rc = download_rows(h, h->s.nodeP + hc.node_off, nullptr, ninv, hc.nn, node_prims))) return rc;
    }
    return GD2D_OK;
}

// Buffers of the one-function-at-a-time entry points, allocated on first use.
static int split_buffers(gd2d_handle *h) {
    if (h->mixed) return fail(h, GD2D_ERR_STATE, "the single-function entry points run the FP64 path only");
    if (!h->state_ready) return fail(h, GD2D_ERR_STATE, "gd2d_set_state must be called for every case first");
    if (!h->split_unew) {
        CUDA_TRY(h, h->buf.alloc(&h->split_unew, (size_t)h->m.Nc));
        CUDA_TRY(h, h->buf.alloc(&h->split_flux, (size_t)h->m.Nc));
        CUDA_TRY(h, h->buf.alloc(&h->split_delta, (size_t)h->m.Nc));
        CUDA_TRY(h, h->buf.alloc(&h->split_diff, (size_t)h->m.Nc));
        CUDA_TRY(h, cudaDeviceSynchronize());
    }
    return GD2D_OK;
}

// A per-cell double4 field of one case to an (nCells x 4) column-major host
// matrix in reference order.
static int download_cells(gd2d_handle *h, int32_t icase, const double4 *src, double *dst) {
    const HostCase &hc = h->cases[icase];
    return download_rows(h, src + hc.cell_off, nullptr, h->d_inv + hc.ref_off, hc.nc, dst);
}

int gd2d_calc_one_stage(gd2d_handle *h, int32_t icase, double beta, double dt, double flow_time, double *fluxes,
                        double *unew) {
    int rc = ensure_case(h, icase);
    if (rc) return rc;
    if ((rc = split_buffers(h))) return rc;
    cudaSetDevice(h->device);
    CUDA_TRY(h, launch_stage_only_f64(h->m, h->s, h->flux, h->quads, beta, dt, flow_time,
                                      h->split_diff_valid ? h->split_diff : nullptr, h->split_unew, h->split_flux,
                                      h->lc, h->stream));
    if ((rc = download_cells(h, icase, h->split_flux, fluxes))) return rc;
    if ((rc = download_cells(h, icase, h->split_unew, unew))) return rc;
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->split_stage_done = true;
    return GD2D_OK;
}

int gd2d_update_variables(gd2d_handle *h, int32_t icase, double *delta) {
    int rc = ensure_case(h, icase);
    if (rc) return rc;
    if ((rc = split_buffers(h))) return rc;
    if (!h->split_stage_done) return fail(h, GD2D_ERR_STATE, "gd2d_calc_one_stage must run first");
    cudaSetDevice(h->device);
    CUDA_TRY(h, launch_update_only_f64(h->m, h->s, h->split_unew, h->split_delta, h->lc, h->stream));
    h->split_stage_done = false;
    h->split_diff_valid = false;
    return download_cells(h, icase, h->split_delta, delta);
}

int gd2d_cells_to_nodes(gd2d_handle *h) {
    if (!h) return fail(nullptr, GD2D_ERR_ARG, "NULL handle");
    int rc = split_buffers(h);
    if (rc) return rc;
    cudaSetDevice(h->device);
    CUDA_TRY(h, launch_node_avg_f64(h->m, h->s, h->visc, false, false, 0, h->m.Nn, 0, 0, false, h->lc, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return GD2D_OK;
}

int gd2d_calc_diff_term(gd2d_handle *h, int32_t icase, double *diff) {
    int rc = ensure_case(h, icase);
    if (rc) return rc;
    if ((rc = split_buffers(h))) return rc;
    if (!h->visc) return fail(h, GD2D_ERR_STATE, "the handle was set up without a viscosity model");
    cudaSetDevice(h->device);
    CUDA_TRY(h, launch_visc_grad_f64(h->m, h->s, h->lc, h->stream));
    CUDA_TRY(h, launch_diff_only_f64(h->m, h->s, h->split_diff, h->lc, h->stream));
    h->split_diff_valid = true;
    return download_cells(h, icase, h->split_diff, diff);
}
// ------------------------------------------------------------ autotuner

namespace {

struct Region {
    void *p;
    size_t bytes;
};

// Every device array a step reads before writing or leaves behind for the
// next step: saving and restoring these makes trial steps invisible.
std::vector<Region> step_state(const gd2d_handle *h) {
    const DevState &s = h->s;
    const DevMesh &m = h->m;
    std::vector<Region> r;
    auto add = [&](const void *p, size_t b) {
        if (p && b) r.push_back({const_cast<void *>(p), b});
    };
    add(s.U, sizeof(double4) * m.Nc);
    add(s.prim, sizeof(double4) * 2 * m.Nc);
    add(s.nodeP, sizeof(double4) * m.Nn);
    add(s.nodeC, sizeof(double4) * m.Nn);
    add(s.g1, sizeof(NodeGrad) * m.Nc);
    add(s.nodeG, sizeof(NodeGrad) * m.Nn);
    add(s.primf, sizeof(float4) * 2 * m.Nc);
    add(s.nodePf, sizeof(float4) * m.Nn);
    add(s.nodeCf, sizeof(float4) * m.Nn);
    add(s.g1f, sizeof(NodeGradF) * m.Nc);
    add(s.nodeGf, sizeof(NodeGradF) * m.Nn);
    add(s.part, sizeof(double) * m.ntiles * kPartials);
    add(s.cstate, sizeof(CaseState) * m.ncases);
    add(s.ring, sizeof(DevStats) * s.ring_len * m.ncases);
    add(s.parity, sizeof(int32_t));
    add(s.node_done, sizeof(unsigned int));
    add(s.gpart, sizeof(double) * h->ngroups * kPartials);
    add(h->Facc, sizeof(double4) * m.Nc);
    add(h->Fslot, sizeof(double4) * m.nfmax * m.Nc);
    return r;
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

cudaError_t copy_regions(const std::vector<Region> &reg, char *snap, bool save, cudaStream_t st) {
    size_t off = 0;
    for (const Region &r : reg) {
        cudaError_t e = save ? cudaMemcpyAsync(snap + off, r.p, r.bytes, cudaMemcpyDeviceToDevice, st)
                             : cudaMemcpyAsync(r.p, snap + off, r.bytes, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return e;
        off += align256(r.bytes);
    }
    return cudaSuccess;
}

}  // namespace

// Device time per step of the handle's current launch shape: restore the
// saved state, one untimed graph (warm-up), restore, then `reps` timed graphs.
static int time_shape(gd2d_handle *h, const std::vector<Region> &reg, char *snap, int reps, double *ms_per_step) {
    const int G = h->graph_steps;
    int rc = G > 1 ? capture_graph(h, G, false) : (drop_graph(h), GD2D_OK);
    if (rc) return rc;
    auto run = [&](int n) -> cudaError_t {
        for (int q = 0; q < n; ++q) {
            cudaError_t e = G > 1 ? cudaGraphLaunch(h->graph, h->stream) : launch_step_kernels(h, nullptr, nullptr);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    CUDA_TRY(h, copy_regions(reg, snap, false, h->stream));
    CUDA_TRY(h, run(1));
    CUDA_TRY(h, copy_regions(reg, snap, false, h->stream));
    CUDA_TRY(h, cudaEventRecord(h->ev_total[0], h->stream));
    CUDA_TRY(h, run(reps));
    CUDA_TRY(h, cudaEventRecord(h->ev_total[1], h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    float ms = 0.f;
    CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev_total[0], h->ev_total[1]));
    *ms_per_step = (double)ms / ((double)reps * G);
    return GD2D_OK;
}

int gd2d_autotune(gd2d_handle *h, int32_t steps_per_trial, gd2d_launch *chosen) {
    if (!h) return fail(nullptr, GD2D_ERR_ARG, "NULL handle");
    if (!h->state_ready) return fail(h, GD2D_ERR_STATE, "gd2d_set_state must be called for every case first");
    if (steps_per_trial <= 0) steps_per_trial = 64;
    cudaSetDevice(h->device);
    const std::vector<Region> reg = step_state(h);
    size_t total = 0;
    for (const Region &r : reg) total += align256(r.bytes);
    char *snap = nullptr;
    {
        cudaError_t e = cudaMalloc((void **)&snap, total);
        if (e != cudaSuccess) return fail(h, GD2D_ERR_OOM, "autotune snapshot of %zu bytes: %s", total,
                                          cudaGetErrorString(e));
    }
    {
        // a failed save must not leak the snapshot buffer
        cudaError_t e = copy_regions(reg, snap, true, h->stream);
        if (e != cudaSuccess) {
            cudaFree(snap);
            return fail(h, GD2D_ERR_CUDA, "autotune save: %s", cudaGetErrorString(e));
        }
    }
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, h->device);
    const LaunchCfg lc0 = h->lc;
    const int G0 = h->graph_steps;
    auto set_shape = [&](const LaunchCfg &lc, int G) {
        h->lc = lc;
        h->lc.grid = dev_sms * lc.min_blocks * (256 / lc.block);
        h->graph_steps = G;
    };
    auto trial = [&](const LaunchCfg &lc, int G, double *ms) {
        set_shape(lc, G);
        const int reps = std::max(1, (steps_per_trial + G - 1) / G);
        return time_shape(h, reg, snap, reps, ms);
    };
    LaunchCfg best = lc0;
    int bestG = G0;
    double best_ms = 0.0;
    int rc = trial(best, bestG, &best_ms);
    // coordinate search: register budget x persistence, then node-pass block,
    // then steps per graph
    for (int mb = 2; rc == GD2D_OK && mb <= 4; ++mb) {
        for (int pers = 0; rc == GD2D_OK && pers <= 1; ++pers) {
            LaunchCfg c = best;
            c.min_blocks = mb;
            c.persistent = pers;
            if (c.min_blocks == best.min_blocks && c.persistent == best.persistent) continue;
            double ms = 0.0;
            rc = trial(c, bestG, &ms);
            if (rc == GD2D_OK && ms < best_ms) { best = c; best_ms = ms; }
        }
    }
    for (int nb : {64, 128, 256}) {
        if (rc != GD2D_OK || nb == best.node_block) continue;
        LaunchCfg c = best;
        c.node_block = nb;
        double ms = 0.0;
        rc = trial(c, bestG, &ms);
        if (rc == GD2D_OK && ms < best_ms) { best = c; best_ms = ms; }
    }
    // a graph length the caller set in the launch record is kept
    for (int G : {8, 32, 128}) {
        if (h->launch.graph_steps > 0) break;
        if (rc != GD2D_OK || G == bestG || G > h->s.ring_len) continue;
        double ms = 0.0;
        rc = trial(best, G, &ms);
        if (rc == GD2D_OK && ms < best_ms) { bestG = G; best_ms = ms; }
    }
    // put the state back whatever happened; on failure keep the old shape
    drop_graph(h);
    cudaError_t e = copy_regions(reg, snap, false, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(snap);
    if (rc != GD2D_OK) {
        set_shape(lc0, G0);
        return rc;
    }
    if (e != cudaSuccess) {
        set_shape(lc0, G0);
        return fail(h, GD2D_ERR_CUDA, "autotune restore: %s", cudaGetErrorString(e));
    }
    set_shape(best, bestG);
    h->launch.min_blocks = best.min_blocks;
    h->launch.persistent = best.persistent;
    h->launch.node_block = best.node_block;
    h->launch.graph_steps = bestG;
    h->last_total_ms = best_ms;
    if (chosen) *chosen = h->launch;
    return GD2D_OK;
}

int gd2d_last_timing(gd2d_handle *h, double *total_ms, double *cell_kernel_ms, int64_t *launches) {
    if (!h) return fail(nullptr, GD2D_ERR_ARG, "NULL handle");
    if (total_ms) *total_ms = h->last_total_ms;
    if (cell_kernel_ms) *cell_kernel_ms = h->last_cell_ms;
    if (launches) *launches = h->last_launches;
    return GD2D_OK;
}

int gd2d_destroy(gd2d_handle *h) {
    if (!h) return GD2D_OK;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    drop_graph(h);
    for (auto &e : h->ev_total) if (e) cudaEventDestroy(e);
    for (auto &e : h->ev_eager) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : h->slice_ev) cudaEventDestroy(e);
    if (h->ring_host) cudaFreeHost(h->ring_host);
    if (h->h_stage) cudaFreeHost(h->h_stage);
    h->buf.free_all();
    if (h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
    return GD2D_OK;
}

}  // extern "C"
