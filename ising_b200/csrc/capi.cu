// capi.cu -- the extern "C" entry points of libisinggpu (declared in include/ising_gpu.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "internal.h"
#include "ensembles.h"
#include "learned.h"

// ======================================================================= errors
namespace isg {
static thread_local std::string g_err;
void set_error(const std::string& m) { g_err = m; }
int fail(int status, const std::string& m) { g_err = m; return status; }
int cuda_fail(cudaError_t e, const char* what) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return ISING_ERR_CUDA;
}
}  // namespace isg

using namespace isg;

#define ISG_TRY(expr)                  \
    do {                               \
        int st_ = (expr);              \
        if (st_ != ISING_OK) return st_; \
    } while (0)

extern "C" const char* ising_last_error(void) { return isg::g_err.c_str(); }

extern "C" const char* ising_status_string(int s) {
    switch (s) {
        case ISING_OK: return "ok";
        case ISING_ERR_ARG: return "invalid argument";
        case ISING_ERR_NAN: return "NaN encountered";
        case ISING_ERR_BOUNDS: return "index out of bounds";
        case ISING_ERR_TIMEOUT: return "device wait timed out";
        case ISING_ERR_UNSUPPORTED: return "unsupported option";
        case ISING_ERR_CUDA: return "CUDA error";
        case ISING_ERR_ALLOC: return "allocation failed";
        case ISING_ERR_LATTICE: return "lattice error";
        case ISING_ERR_CAPACITY: return "stack capacity exceeded";
        default: return "unknown status";
    }
}

extern "C" const char* ising_version(void) { return "isinggpu 0.1 sm_100a"; }

// ======================================================================= helpers
namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

template <typename T>
int dev_alloc(T** p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) return fail(ISING_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return ISING_OK;
}

// status word -> error code; clears it
int check_status(ising_mesh* m) {
    ISG_CUDA(cudaMemcpyAsync(m->h_pinned, m->d_status, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    ISG_CUDA(cudaStreamSynchronize(m->stream));
    int st;
    std::memcpy(&st, m->h_pinned, sizeof(int));
    if (st) {
        ISG_CUDA(cudaMemsetAsync(m->d_status, 0, sizeof(int), m->stream));
        if (st & kStatNan) return fail(ISING_ERR_NAN, "NaN in spins or proposals");
        if (st & kStatTimeout) return fail(ISING_ERR_TIMEOUT, "device wait timed out");
        if (st & kStatBounds) return fail(ISING_ERR_BOUNDS, "device index out of bounds");
    }
    return ISING_OK;
}

int validate_params(const ising_params* p) {
    if (!p) return fail(ISING_ERR_ARG, "params is NULL");
    const double v[] = {p->J, p->J_prime, p->Dz, p->Dz_prime, p->B, p->K, p->zeeman_factor};
    for (double x : v) if (!std::isfinite(x)) return fail(ISING_ERR_NAN, "non-finite Hamiltonian parameter");
    if (p->dmi_mode != ISING_DMI_INTERFACIAL && p->dmi_mode != ISING_DMI_BULK)
        return fail(ISING_ERR_ARG, "dmi_mode must be ISING_DMI_INTERFACIAL or ISING_DMI_BULK");
    return ISING_OK;
}

// DMI vector of a bond with min-image r = r_j - r_i, reference orientation r_hat = -r/|r|
// (src/energyMin.f90:135-138).
void bond_dmi(const Lattice& L, const ising_params& p, const double r[3], double D[3]) {
    const double n = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    const double rh[3] = {-r[0] / n, -r[1] / n, -r[2] / n};
    if (p.dmi_mode == ISING_DMI_BULK) {
        for (int k = 0; k < 3; ++k) D[k] = p.Dz * rh[k];
        return;
    }
    double ax[3] = {p.dmi_axis[0], p.dmi_axis[1], p.dmi_axis[2]};
    if (ax[0] == 0.0 && ax[1] == 0.0 && ax[2] == 0.0) {
        const double cn = std::sqrt(L.cv[0] * L.cv[0] + L.cv[1] * L.cv[1] + L.cv[2] * L.cv[2]);
        for (int k = 0; k < 3; ++k) ax[k] = L.cv[k] / cn;
    }
    const double t[3] = {p.Dz * ax[0], p.Dz * ax[1], p.Dz * ax[2]};
    D[0] = t[1] * rh[2] - t[2] * rh[1];
    D[1] = t[2] * rh[0] - t[0] * rh[2];
    D[2] = t[0] * rh[1] - t[1] * rh[0];
}

HamDev make_ham(const ising_params& p) {
    HamDev h{};
    h.J = (float)p.J;
    h.Jp = (float)p.J_prime;
    h.Bz = (float)(p.zeeman_factor * p.B);
    h.K = (float)p.K;
    h.kx = (float)p.K_axis[0]; h.ky = (float)p.K_axis[1]; h.kz = (float)p.K_axis[2];
    return h;
}

bool uses_shell2(const Lattice& L, const ising_params& p) {
    return p.include_Jp && p.J_prime != 0.0 && L.nshells > 1;
}

// Fill the device stencil of `m` for the given Hamiltonian.  legacy: the legacy list with
// (J, D); otherwise shell 1 with (J, D) and shell 2 with J' when active.
int upload_stencil(ising_mesh* m, const ising_params& p, bool legacy, Slot* dst_slots, int* dst_count) {
    // one stencil builder for every path (the allocation-free energy entry point fills the
    // same tables into its own host memory)
    std::vector<Slot> slots((size_t)kMaxSub * kMaxSlots);
    std::vector<int> cnt(kMaxSub, 0);
    ISG_TRY(fill_query_stencil_host(m, p, legacy, slots.data(), cnt.data()));
    ISG_CUDA(cudaMemcpyAsync(dst_slots, slots.data(), slots.size() * sizeof(Slot), cudaMemcpyHostToDevice, m->stream));
    ISG_CUDA(cudaMemcpyAsync(dst_count, cnt.data(), cnt.size() * sizeof(int), cudaMemcpyHostToDevice, m->stream));
    // the host vectors die at return: make the copies complete first
    ISG_CUDA(cudaStreamSynchronize(m->stream));
    return ISING_OK;
}

// the mesh's query stencil (local energies, reductions); sweeps of a PT own theirs
int upload_query_stencil(ising_mesh* m, const ising_params& p, bool legacy) {
    return upload_stencil(m, p, legacy, m->d_slots, m->d_slot_count);
}
StencilDev stencil_of(const ising_mesh* m) { return StencilDev{m->d_slots, m->d_slot_count, m->lat.nsub}; }

// SC fast path: D vectors per direction (+x,-x,+y,-y,+z,-z) and the specialisation kind.
int sc_dmi(const ising_mesh* m, const ising_params& p, HamDev* h, int* kind) {
    const Lattice& L = m->lat;
    for (const auto& q : L.shell[0][0]) {
        int k = q.dx == 1 ? 0 : q.dx == -1 ? 1 : q.dy == 1 ? 2 : q.dy == -1 ? 3 : q.dz == 1 ? 4 : 5;
        double D[3] = {0, 0, 0};
        if (p.Dz != 0.0) bond_dmi(L, p, q.r, D);
        for (int c = 0; c < 3; ++c) h->D[k][c] = (float)D[c];
    }
    if (p.Dz == 0.0) { *kind = 0; return ISING_OK; }
    const float d = (float)p.Dz;
    auto eq = [](const float* a, float x, float y, float z) { return a[0] == x && a[1] == y && a[2] == z; };
    const bool bulk = eq(h->D[0], -d, 0, 0) && eq(h->D[1], d, 0, 0) && eq(h->D[2], 0, -d, 0) &&
                      eq(h->D[3], 0, d, 0) && eq(h->D[4], 0, 0, -d) && eq(h->D[5], 0, 0, d);
    const bool intz = eq(h->D[0], 0, -d, 0) && eq(h->D[1], 0, d, 0) && eq(h->D[2], d, 0, 0) &&
                      eq(h->D[3], -d, 0, 0) && eq(h->D[4], 0, 0, 0) && eq(h->D[5], 0, 0, 0);
    // eq() compares exact floats; -0.0f == 0.0f holds, so sign-of-zero does not matter
    *kind = bulk ? 1 : intz ? 2 : 3;
    return ISING_OK;
}

// Colour classes of a mesh that is not on the checkerboard path.  Octant-layout meshes: sets
// of blocks (cell octant, sublattice), the fewer of (1) the octant classes (octant o,
// sublattice group g) as class o * groups + g, or without J', where the mesh has them, its
// shell-1 classes (every octant of each), and (2) a DSatur colouring of the block graph of the
// active shells; else a greedy colouring of the active shells' bonds.
int host_colouring(ising_mesh* m, bool shell2, Colouring& c) {
    if (!c.host_colour.empty()) return ISING_OK;
    const Lattice& L = m->lat;
    if (m->layout.cb == 2) {
        auto code = [&](int o, int rank) { return (uint8_t)((o << 4) | rank); };
        std::vector<std::vector<uint8_t>> cls;
        if (!shell2 && !m->oct_class0.empty()) {
            for (size_t k = 0; k + 1 < m->oct_class0.size(); ++k) {
                cls.emplace_back();
                for (int o = 0; o < 8; ++o)
                    for (int r = m->oct_class0[k]; r < m->oct_class0[k + 1]; ++r) cls.back().push_back(code(o, r));
            }
        } else {
            const int ng = (int)m->oct_rank0.size() - 1;
            for (int k = 0; k < 8 * ng; ++k) {
                cls.emplace_back();
                for (int r = m->oct_rank0[k % ng]; r < m->oct_rank0[k % ng + 1]; ++r) cls.back().push_back(code(k / ng, r));
            }
        }
        std::vector<std::vector<int>> ds;
        if (octant_block_classes(L, shell2, &ds) && ds.size() < cls.size()) {
            cls.clear();
            for (const auto& k : ds) {
                cls.emplace_back();
                for (int v : k) cls.back().push_back(code(v / L.nsub, m->layout.srank[v % L.nsub]));
                std::sort(cls.back().begin(), cls.back().end());
            }
        }
        std::vector<int> of_block(128, -1);
        for (size_t k = 0; k < cls.size(); ++k)
            for (uint8_t b : cls[k]) of_block[b] = (int)k;
        c.host_colour.resize(L.natoms);
        for (int64_t at = 0; at < L.natoms; ++at) {
            int ix, iy, iz, sb;
            L.cell_of(at, &ix, &iy, &iz, &sb);
            const int o = ((ix & 1) << 2) | ((iy & 1) << 1) | (iz & 1);
            c.host_colour[at] = of_block[code(o, m->layout.srank[sb])];
        }
        c.ncol = (int)cls.size();
        c.oct_blocks = std::move(cls);
        return ISING_OK;
    }
    if (m->layout.cb == 3 && !shell2) {   // the two sublattices
        c.host_colour.resize(L.natoms);
        for (int64_t at = 0; at < L.natoms; ++at) c.host_colour[at] = (int)(at % 2);
        c.ncol = 2;
        return ISING_OK;
    }
    int ncol = 0;
    ISG_TRY(greedy_colouring(L, shell2, &c.host_colour, &ncol));
    c.ncol = ncol;
    return ISING_OK;
}

int ensure_colouring(ising_mesh* m, bool shell2, Colouring** out) {
    Colouring& c = m->colour[shell2 ? 1 : 0];
    if (c.d_sites) { *out = &c; return ISING_OK; }
    ISG_TRY(host_colouring(m, shell2, c));
    c.class_start.assign(c.ncol + 1, 0);
    for (int v : c.host_colour) c.class_start[v + 1]++;
    for (int k = 0; k < c.ncol; ++k) c.class_start[k + 1] += c.class_start[k];
    std::vector<int> sites(m->lat.natoms);
    std::vector<int> pos(c.class_start.begin(), c.class_start.end() - 1);
    for (int64_t a = 0; a < m->lat.natoms; ++a) sites[pos[c.host_colour[a]]++] = (int)a;
    ISG_TRY(dev_alloc(&c.d_sites, sites.size()));
    ISG_CUDA(cudaMemcpy(c.d_sites, sites.data(), sites.size() * sizeof(int), cudaMemcpyHostToDevice));
    *out = &c;
    return ISING_OK;
}

// One sweep plan: which kernels to launch for a set of replicas.
struct SweepPlan {
    bool sc = false;
    bool tma = false;          // TMA-staged colour pass (nz % 8 == 0)
    int group = 1;             // replicas per L2 group in the paired schedule
    int dmi_kind = 0;
    HamDev ham{};
    Colouring* col = nullptr;
    int slots_per_rep = 0;
    Slot* d_slots = nullptr;   // general path: stencil buffers this plan reads
    int* d_count = nullptr;
    const float* demag = nullptr;   // general path: demagnetising field of the swept replica
    int oct_maxcnt = 0;        // octant layout: k_octant_fast's table width (0: k_octant_colour)
    bool oct_engine = false;   // octant layout: every sweep of a call in one persistent launch
    int oct_reach = 1;         // its dependency reach in packed x-planes
    int oct_grid = 0;          // its persistent blocks
    bool bip = false;          // layout 3 without J': the two sublattice classes (k_bip_sweep)
    BipClass bipc[2] = {};     // their first-shell bonds
    int oct_stall = 0;         // test hook (ising_pt_inject_stall): the next round's waits run out
    uint64_t oct_wait_ns = 2000000000ull;   // bound of every wait of the engine
};

// Fills plan for Hamiltonian p; the general path uploads its stencil into (slots, count).
int make_plan(ising_mesh* m, const ising_params& p, SweepPlan* plan, Slot* slots, int* count) {
    plan->ham = make_ham(p);
    const bool sh2 = uses_shell2(m->lat, p);
    if (m->layout.cb == 1 && !sh2 && !p.demag) {
        plan->sc = true;
        ISG_TRY(sc_dmi(m, p, &plan->ham, &plan->dmi_kind));
        const Lattice& Lt = m->lat;
        plan->tma = false;   // the register kernel measures faster; the TMA pass is opt-in
        (void)Lt;
        plan->slots_per_rep = std::max(cb_slots_per_rep(), plan->tma ? cb_tma_slots_per_rep(Lt.nx, Lt.ny, Lt.nz) : 0);
        // replicas per group: the two groups of a paired launch stay well inside the 126 MB L2
        const double rep_bytes = 12.0 * (double)m->lat.natoms;
        plan->group = std::max(1, (int)(kL2GroupBytes / rep_bytes));
        return ISING_OK;
    }
    plan->sc = false;
    plan->d_slots = slots;
    plan->d_count = count;
    ISG_TRY(upload_stencil(m, p, false, slots, count));
    ISG_TRY(ensure_colouring(m, sh2, &plan->col));
    int tot = 0;
    if (m->layout.cb == 3 && !sh2 && !p.demag && m->lat.nz % 2 == 0 && m->lat.nz / 2 <= 256) {
        // the first shell of each sublattice as bonds (a, b, c) to the other one
        std::vector<Slot> hs((size_t)kMaxSub * kMaxSlots);
        std::vector<int> hc(kMaxSub, 0);
        ISG_TRY(fill_query_stencil_host(m, p, false, hs.data(), hc.data()));
        bool ok = true;
        for (int sb = 0; sb < 2 && ok; ++sb) {
            BipClass& c = plan->bipc[sb];
            for (int k = 0; k < 3; ++k) c.base[k] = m->bip_base[sb][k];
            int seen = 0;
            ok = hc[sb] == 8;
            for (int q = 0; q < hc[sb] && ok; ++q) {
                const Slot& e = hs[(size_t)sb * kMaxSlots + q];
                const int aa = e.dx - c.base[0], bb = e.dy - c.base[1], cc = e.dz - c.base[2];
                ok = e.sub == 1 - sb && aa >= 0 && aa <= 1 && bb >= 0 && bb <= 1 && cc >= 0 && cc <= 1;
                if (!ok) break;
                const int i = aa * 4 + bb * 2 + cc;
                seen |= 1 << i;
                c.w[i] = e.w; c.D[i][0] = e.Dx; c.D[i][1] = e.Dy; c.D[i][2] = e.Dz;
            }
            ok = ok && seen == 0xff;
        }
        if (ok) {
            plan->bip = true;
            plan->slots_per_rep = 2 * bip_slots_per_class();
            return ISING_OK;
        }
    }
    if (m->layout.cb == 2) {
        // the per-class stencil of k_octant_fast: every packed offset floor((o + d) / 2),
        // o in {0, 1}, must lie within one period of its axis
        std::vector<Slot> hs((size_t)kMaxSub * kMaxSlots);
        std::vector<int> hc(kMaxSub, 0);
        ISG_TRY(fill_query_stencil_host(m, p, false, hs.data(), hc.data()));
        const Lattice& Lt = m->lat;
        const int half[3] = {Lt.nx / 2, Lt.ny / 2, Lt.nz / 2};
        int maxcnt = 0, reach = 0;
        bool fits = true;
        for (int sub = 0; sub < Lt.nsub; ++sub) {
            maxcnt = std::max(maxcnt, hc[sub]);
            for (int q = 0; q < hc[sub]; ++q) {
                const Slot& e = hs[(size_t)sub * kMaxSlots + q];
                const int d[3] = {e.dx, e.dy, e.dz};
                for (int ax = 0; ax < 3; ++ax)
                    for (int o = 0; o < 2; ++o) {
                        const int t = o + d[ax];
                        const int ex = (t - (t & 1)) / 2;
                        if (ex < -half[ax] || ex > half[ax]) fits = false;
                        if (ax == 0) reach = std::max(reach, std::abs(ex));
                    }
            }
        }
        plan->oct_maxcnt = fits ? std::max(maxcnt, 1) : 0;
        // the persistent engine (opt-in, sweep_kernel 3): one partial slot per (replica,
        // packed x-plane); plan->oct_engine is set by the PT object that asks for it
        if (plan->oct_maxcnt > 0) {
            plan->oct_reach = std::max(reach, 1);
            ISG_TRY(octant_engine_grid(&plan->oct_grid));
            if (!m->d_oct_sync)
                ISG_TRY(dev_alloc(&m->d_oct_sync, (size_t)m->n_replicas * (size_t)(Lt.nx / 2) + 2));
        }
        // the classes are lists of blocks (octant, storage rank), host_colouring's
        for (const auto& k : plan->col->oct_blocks)
            tot += octant_class_slots(m->layout.q8, (int)k.size(), plan->oct_maxcnt);
        // every replica in each class launch: L2-sized replica groups (a group running all its
        // sweeps before the next) measured no faster on BCC 96^3 x 16 and much slower on
        // hyper-kagome, whose classes are small; large launches let a thread take several sites
        // (ising_pt_options.l2_group still sets a group size)
        plan->group = INT32_MAX;
        if (plan->oct_maxcnt > 0) tot = std::max(tot, Lt.nx / 2);
    } else {
        for (int k = 0; k < plan->col->ncol; ++k)
            tot += general_slots_for(plan->col->class_start[k + 1] - plan->col->class_start[k]);
    }
    plan->slots_per_rep = tot;
    return ISING_OK;
}

// Checkerboard schedule for n_sweeps sweeps of replicas [rep_first, rep_first + n_rep):
// replica groups g = 0..G-1, first-colour units R_0..R_{M-1} and second-colour units
// B_0..B_{M-1} in (sweep, group) order.  With G >= 2: launch 0 = {R_0}, launch j = {B_{j-1},
// R_j}, launch M = {B_{M-1}}; R_j needs B_{j-G} (same group, previous sweep), finished by
// launch j-G+1 < j, and B_j needs R_j, finished by launch j.  With one group the units run
// one per launch.
int enqueue_cb(ising_mesh* m, const SweepPlan& plan, int rep_first, int n_rep, const double* d_beta_rep,
               uint32_t sw0, int n_sweeps, uint64_t seed, uint32_t ensemble, int move, double r,
               double* partials) {
    const Lattice& L = m->lat;
    CbLaunch a{};
    a.spins = m->d_spins; a.natoms = L.natoms; a.nx = L.nx; a.ny = L.ny; a.nz = L.nz;
    a.beta_rep = d_beta_rep; a.sweep_ctr = m->d_sweep; a.seed = seed; a.ensemble = ensemble; a.r = (float)r;
    a.ham = plan.ham; a.partials = partials; a.slots_per_rep = plan.slots_per_rep; a.status = m->d_status;
    const int G = (n_rep + plan.group - 1) / plan.group;
    auto unit = [&](int j, int colour) {
        const int sw = j / G, g = j % G;
        CbSeg sgm;
        sgm.rep_first = rep_first + g * plan.group;
        sgm.n_rep = std::min(plan.group, rep_first + n_rep - sgm.rep_first);
        sgm.colour = colour;
        sgm.sweep_offset = sw0 + (uint32_t)sw;
        return sgm;
    };
    const int M = G * n_sweeps;
    if (G == 1) {
        for (int j = 0; j < M; ++j)
            for (int c = 0; c < 2; ++c) {
                a.seg[0] = unit(j, c);
                a.seg[1] = CbSeg{0, 0, 0, 0};
                a.n_seg = 1;
                ISG_TRY(plan.tma ? launch_cb_tma(a, move, plan.dmi_kind, m->stream)
                                 : launch_cb_sweep(a, move, plan.dmi_kind, m->stream));
            }
        return ISING_OK;
    }
    for (int j = 0; j <= M; ++j) {
        a.n_seg = 0;
        if (j >= 1) a.seg[a.n_seg++] = unit(j - 1, 1);
        if (j < M) a.seg[a.n_seg++] = unit(j, 0);
        if (a.n_seg == 1) a.seg[1] = CbSeg{0, 0, 0, 0};
        ISG_TRY(plan.tma ? launch_cb_tma(a, move, plan.dmi_kind, m->stream)
                         : launch_cb_sweep(a, move, plan.dmi_kind, m->stream));
    }
    return ISING_OK;
}

// n_sweeps consecutive sweeps (sweep offsets sw0 .. sw0+n_sweeps-1) of replicas
// [rep_first, rep_first + n_rep), all colour classes.
int enqueue_sweeps(ising_mesh* m, const SweepPlan& plan, int rep_first, int n_rep, const double* d_beta_rep,
                   uint32_t sw0, int n_sweeps, uint64_t seed, uint32_t ensemble, int move, double r,
                   double* partials) {
    if (plan.sc)
        return enqueue_cb(m, plan, rep_first, n_rep, d_beta_rep, sw0, n_sweeps, seed, ensemble, move, r, partials);
    const Lattice& L = m->lat;
    GeneralLaunch g{};
    g.spins = m->d_spins + (int64_t)rep_first * 3 * L.natoms;
    g.natoms = L.natoms; g.nx = L.nx; g.ny = L.ny; g.nz = L.nz; g.nsub = L.nsub;
    g.n_rep = n_rep; g.rep_first = rep_first; g.beta_rep = d_beta_rep; g.sweep_ctr = m->d_sweep;
    g.seed = seed; g.ensemble = ensemble; g.move = move; g.r = (float)r;
    philox_round_keys(seed, g.rk);
    g.ham = plan.ham; g.st = StencilDev{plan.d_slots, plan.d_count, L.nsub}; g.layout = m->layout;
    g.partials = partials; g.slots_per_rep = plan.slots_per_rep; g.status = m->d_status;
    g.demag = plan.demag; g.mu0 = (float)kMu0;
    if (m->layout.cb == 3 && plan.bip) {   // the two sublattice classes
        for (int sw = 0; sw < n_sweeps; ++sw) {
            g.sweep_offset = sw0 + (uint32_t)sw;
            for (int sb = 0; sb < 2; ++sb) {
                g.slot_base = sb * bip_slots_per_class();
                ISG_TRY(launch_bip_sweep(g, plan.bipc[sb], sb, m->stream));
            }
        }
        return ISING_OK;
    }
    if (m->layout.cb == 2 && plan.oct_engine) {   // every sweep of the call in one launch
        OctEngineLaunch e{};
        const int hx = L.nx / 2;
        e.head = m->d_oct_sync;
        e.abort = m->d_oct_sync + 1;
        e.done = m->d_oct_sync + 2;
        e.n_sweeps = n_sweeps;
        const auto& cls = plan.col->oct_blocks;
        e.ncls = (int)cls.size();
        e.maxnb = 0;
        int nb = 0;
        for (int c = 0; c < e.ncls; ++c) {
            e.start[c] = (uint8_t)nb;
            for (uint8_t b : cls[c]) e.code[nb++] = b;
            e.maxnb = std::max(e.maxnb, (int)cls[c].size());
        }
        e.start[e.ncls] = (uint8_t)nb;
        e.reach = plan.oct_reach;
        e.wait_ns = plan.oct_wait_ns;
        e.stall = plan.oct_stall;
        e.grid = plan.oct_grid;
        g.oct_maxcnt = plan.oct_maxcnt;
        g.sweep_offset = sw0;
        g.slot_base = 0;
        ISG_CUDA(cudaMemsetAsync(m->d_oct_sync, 0, ((size_t)n_rep * hx + 2) * sizeof(uint32_t), m->stream));
        return launch_octant_engine(g, e, m->stream);
    }
    if (m->layout.cb == 2) {   // octant classes: lists of blocks (octant, storage rank)
        // replicas are independent: each L2-sized group of replicas runs all its sweeps
        // (every class, in order) before the next group starts, so a group's spins stay in L2
        g.oct_maxcnt = plan.oct_maxcnt;
        const auto& cls = plan.col->oct_blocks;
        const int G = std::max(1, plan.group);
        for (int gr = 0; gr < n_rep; gr += G) {
            g.rep_first = rep_first + gr;
            g.n_rep = std::min(G, n_rep - gr);
            g.spins = m->d_spins + (int64_t)g.rep_first * 3 * L.natoms;
            for (int sw = 0; sw < n_sweeps; ++sw) {
                g.sweep_offset = sw0 + (uint32_t)sw;
                int slot = 0;
                for (const auto& k : cls) {
                    OctBlocks bl{};
                    bl.n = (int)k.size();
                    for (int i = 0; i < bl.n; ++i) bl.code[i] = k[i];
                    g.slot_base = slot;
                    ISG_TRY(launch_octant_class(g, bl, m->stream));
                    slot += octant_class_slots(m->layout.q8, bl.n, plan.oct_maxcnt);
                }
            }
        }
        return ISING_OK;
    }
    for (int sw = 0; sw < n_sweeps; ++sw) {
        g.sweep_offset = sw0 + (uint32_t)sw;
        int slot = 0;
        for (int k = 0; k < plan.col->ncol; ++k) {
            g.sites = plan.col->d_sites + plan.col->class_start[k];
            g.n_sites = plan.col->class_start[k + 1] - plan.col->class_start[k];
            g.slot_base = slot;
            ISG_TRY(launch_general_colour(g, m->stream));
            slot += general_slots_for(g.n_sites);
        }
    }
    return ISING_OK;
}

int enqueue_sweep(ising_mesh* m, const SweepPlan& plan, int rep_first, int n_rep, const double* d_beta_rep,
                  uint32_t sweep_offset, uint64_t seed, uint32_t ensemble, int move, double r, double* partials) {
    return enqueue_sweeps(m, plan, rep_first, n_rep, d_beta_rep, sweep_offset, 1, seed, ensemble, move, r, partials);
}

int check_replica_only(const ising_mesh* m, int replica) {
    if (!m) return fail(ISING_ERR_ARG, "mesh is NULL");
    if (m->device < 0) return fail(ISING_ERR_ARG, "mesh was created without a device (device = -1)");
    if (replica < 0 || replica >= m->n_replicas) return fail(ISING_ERR_BOUNDS, "replica index out of range");
    return ISING_OK;
}
// the replica check of every synchronous entry point: also lets pending transfers land
int check_replica(const ising_mesh* m, int replica) {
    ISG_TRY(check_replica_only(m, replica));
    return mesh_settle(m);
}

// energy + magnetisation of replicas [first, first+n) into d_out[n][4] (device)
int enqueue_energy(ising_mesh* m, const ising_params& p, int first, int n, double* d_out, double* d_tmp) {
    ISG_TRY(upload_query_stencil(m, p, p.legacy_neighbours != 0));
    ReduceLaunch a{};
    a.spins = m->d_spins + (int64_t)first * 3 * m->lat.natoms;
    a.natoms = m->lat.natoms; a.nx = m->lat.nx; a.ny = m->lat.ny; a.nz = m->lat.nz; a.nsub = m->lat.nsub;
    a.n_rep = n; a.ham = make_ham(p); a.st = stencil_of(m); a.layout = m->layout; a.out = d_out; a.block_tmp = d_tmp;
    a.blocks_per_rep = energy_blocks_for(m->lat.natoms);
    return launch_energy_mag(a, m->stream);
}

int energy_tmp_doubles(const ising_mesh* m, int n) { return energy_blocks_for(m->lat.natoms) * n * 4; }

}  // namespace

// ======================================================================= unit cells
extern "C" int ising_unit_cell(int kind, double* a, double* b, double* c, double* ab, double* bc,
                               double* ca, float* frac, int* n) {
    if (!a || !b || !c || !ab || !bc || !ca || !frac || !n) return fail(ISING_ERR_ARG, "NULL argument");
    *ab = *bc = *ca = 90.0;
    if (kind == ISING_CELL_SC) {
        *a = *b = *c = 1.0;
        frac[0] = frac[1] = frac[2] = 0.f;
        *n = 1;
        return ISING_OK;
    }
    if (kind == ISING_CELL_BCC) {  // src/unit_cells.f90:21-28
        *a = *b = *c = 2.0;
        const float f[6] = {0.f, 0.f, 0.f, 0.5f, 0.5f, 0.5f};
        std::memcpy(frac, f, sizeof f);
        *n = 2;
        return ISING_OK;
    }
    if (kind == ISING_CELL_HYPER_KAGOME) {  // src/unit_cells.f90:47-76
        *a = *b = *c = 6.0;
        const float f[36] = {-0.5f, 0.0f, 0.5f,   -0.25f, 0.75f, 0.5f,  -0.5f, 0.75f, 0.25f,
                             -0.25f, 0.25f, 0.0f, -0.5f, 0.25f, 0.75f,  -0.25f, 0.5f, 0.75f,
                             -0.75f, 0.5f, 0.25f, 0.0f, 0.5f, 0.5f,     0.0f, 0.25f, 0.25f,
                             -0.75f, 0.75f, 0.0f, 0.0f, 0.0f, 0.0f,     -0.75f, 0.0f, 0.75f};
        std::memcpy(frac, f, sizeof f);
        *n = 12;
        return ISING_OK;
    }
    return fail(ISING_ERR_ARG, "unknown unit cell kind");
}

// ======================================================================= mesh
extern "C" int ising_mesh_create(const float* frac, int nsub, int nx, int ny, int nz, double a, double b,
                                 double c, double ab, double bc, double ca, double shell_tol, int n_shells,
                                 int n_replicas, int device, ising_mesh** out) {
    if (!out) return fail(ISING_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (n_replicas < 1) return fail(ISING_ERR_ARG, "n_replicas must be >= 1");
    std::unique_ptr<ising_mesh> m(new ising_mesh());
    ISG_TRY(build_lattice(frac, nsub, nx, ny, nz, a, b, c, ab, bc, ca, shell_tol, n_shells, &m->lat));
    m->checkerboard = is_checkerboard_sc(m->lat);
    {
        const Lattice& L = m->lat;
        m->layout = Layout{m->checkerboard && L.nz % 4 == 0 ? 1 : 0, L.nx, L.ny, L.nz, L.nsub, L.natoms / 2};
        std::vector<int> grp, cls;
        int ng = 0;
        // two sublattices joined only to each other (BCC): sublattice planes; other crystals:
        // octant order when the octant colouring applies (ranks grouped by sublattice group,
        // so each colour class is one contiguous range)
        if (!m->checkerboard && bipartite_pair(L, m->bip_base)) {
            m->layout.cb = 3;
        } else if (!m->checkerboard && octant_groups(L, &grp, &ng, &cls)) {
            m->layout.cb = 2;
            m->layout.q8 = L.ncells / 8;
            int next = 0;
            m->oct_rank0.assign(1, 0);
            m->oct_class0.clear();
            for (int g = 0; g < ng; ++g) {
                if (!cls.empty() && (g == 0 || cls[g] != cls[g - 1])) m->oct_class0.push_back(next);
                for (int sb = 0; sb < L.nsub; ++sb)
                    if (grp[sb] == g) {
                        m->layout.srank[sb] = (uint8_t)next;
                        m->layout.sofr[next] = (uint8_t)sb;
                        ++next;
                    }
                m->oct_rank0.push_back(next);
            }
            if (!cls.empty()) m->oct_class0.push_back(next);
        }
    }
    if (device == -1) {  // lattice tables only
        m->device = -1;
        m->n_replicas = n_replicas;
        *out = m.release();
        return ISING_OK;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(ISING_ERR_CUDA, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(ISING_ERR_ARG, "device index out of range");
    DeviceGuard g(device);
    m->device = device;
    m->n_replicas = n_replicas;
    ISG_CUDA(cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking));
    m->stream = m->own_stream;
    const int64_t N = m->lat.natoms;
    ISG_TRY(dev_alloc(&m->d_spins, (size_t)n_replicas * 3 * N));
    ISG_TRY(dev_alloc(&m->d_sweep, n_replicas));
    ISG_TRY(dev_alloc(&m->d_beta, n_replicas));
    ISG_TRY(dev_alloc(&m->d_scratch, kScratchDoubles));
    ISG_TRY(dev_alloc(&m->d_status, 1));
    ISG_TRY(dev_alloc(&m->d_slots, (size_t)kMaxSub * kMaxSlots));
    ISG_TRY(dev_alloc(&m->d_slot_count, kMaxSub));
    ISG_TRY(dev_alloc(&m->d_plaq, 16));
    ISG_TRY(dev_alloc(&m->d_winding_tmp, (size_t)n_replicas * nz));
    ISG_CUDA(cudaMallocHost((void**)&m->h_pinned, kScratchDoubles * sizeof(double)));
    ISG_CUDA(cudaMemset(m->d_spins, 0, (size_t)n_replicas * 3 * N * sizeof(float)));
    ISG_CUDA(cudaMemset(m->d_sweep, 0, n_replicas * sizeof(uint32_t)));
    ISG_CUDA(cudaMemset(m->d_status, 0, sizeof(int)));
    m->h_sweep.assign(n_replicas, 0u);
    // winding plaquette: s1 = first atom of the cell (last unit-cell atom, linked-list head,
    // src/chainMesh.f90:663-671), s2 = +a of s1, s4 = +b of s2, s3 = +b of s1 (rsp:344-347)
    {
        const Lattice& L = m->lat;
        const int s1 = L.nsub - 1;
        const NbrSlot& a2 = L.deriv[s1 * 6 + 0 * 2 + 1];
        const NbrSlot& a4 = L.deriv[a2.sub * 6 + 1 * 2 + 1];
        const NbrSlot& a3 = L.deriv[s1 * 6 + 1 * 2 + 1];
        const int plaq[16] = {0, 0, 0, s1,
                              a2.dx, a2.dy, a2.dz, a2.sub,
                              a2.dx + a4.dx, a2.dy + a4.dy, a2.dz + a4.dz, a4.sub,
                              a3.dx, a3.dy, a3.dz, a3.sub};
        ISG_CUDA(cudaMemcpy(m->d_plaq, plaq, sizeof plaq, cudaMemcpyHostToDevice));
    }
    *out = m.release();
    return ISING_OK;
}

namespace {
void xfer_release(ising_mesh* m);   // asynchronous-transfer state (defined with ising_spins_*_async)
}

extern "C" int ising_mesh_destroy(ising_mesh* m) {
    if (!m) return ISING_OK;
    if (m->device < 0) { delete m; return ISING_OK; }
    DeviceGuard g(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    xfer_release(m);
    cudaFree(m->d_spins); cudaFree(m->d_sweep); cudaFree(m->d_scratch); cudaFree(m->d_status);
    cudaFree(m->d_staging); cudaFree(m->d_beta); cudaFree(m->d_winding_tmp); cudaFree(m->d_slots); cudaFree(m->d_slot_count);
    cudaFree(m->d_plaq); cudaFree(m->d_oct_sync);
    isg::skyrmion_release(m);
    isg::demag_release(m);
    for (auto& c : m->colour) cudaFree(c.d_sites);
    if (m->h_pinned) cudaFreeHost(m->h_pinned);
    if (m->own_stream) cudaStreamDestroy(m->own_stream);
    delete m;
    return ISING_OK;
}

extern "C" int ising_mesh_get_info(const ising_mesh* m, ising_mesh_info* info) {
    if (!m || !info) return fail(ISING_ERR_ARG, "NULL argument");
    const Lattice& L = m->lat;
    std::memset(info, 0, sizeof *info);
    info->num_atoms = L.natoms; info->num_cells = L.ncells;
    info->nx = L.nx; info->ny = L.ny; info->nz = L.nz; info->n_sub = L.nsub;
    info->n_shells = L.nshells; info->n_replicas = m->n_replicas;
    info->shell_size[0] = (int)L.shell[0][0].size();
    info->shell_size[1] = (int)L.shell[1][0].size();
    info->checkerboard = m->layout.cb;
    for (int k = 0; k < 3; ++k) { info->a_vec[k] = L.av[k]; info->b_vec[k] = L.bv[k]; info->c_vec[k] = L.cv[k]; }
    return ISING_OK;
}

extern "C" int ising_mesh_set_stream(ising_mesh* m, void* stream) {
    if (!m) return fail(ISING_ERR_ARG, "mesh is NULL");
    if (m->device < 0) return fail(ISING_ERR_ARG, "mesh was created without a device (device = -1)");
    DeviceGuard g(m->device);
    ISG_TRY(mesh_settle(m));
    // order the switch: work already issued on the old stream completes first
    ISG_CUDA(cudaStreamSynchronize(m->stream));
    m->stream = stream ? static_cast<cudaStream_t>(stream) : m->own_stream;
    return ISING_OK;
}

extern "C" int ising_mesh_positions(const ising_mesh* m, float* xyz) {
    if (!m || !xyz) return fail(ISING_ERR_ARG, "NULL argument");
    for (int64_t a = 0; a < m->lat.natoms; ++a) m->lat.position(a, xyz + 3 * a);
    return ISING_OK;
}

extern "C" int ising_mesh_neighbours(const ising_mesh* m, int64_t atom, int shell, int64_t* out, int cap, int* n) {
    if (!m || !n) return fail(ISING_ERR_ARG, "NULL argument");
    const Lattice& L = m->lat;
    if (atom < 0 || atom >= L.natoms) return fail(ISING_ERR_BOUNDS, "atom index out of range");
    if (shell < -1 || shell > 1) return fail(ISING_ERR_ARG, "shell must be -1, 0 or 1");
    int ix, iy, iz, s;
    L.cell_of(atom, &ix, &iy, &iz, &s);
    const auto& lst = shell < 0 ? L.legacy[s] : L.shell[shell][s];
    *n = (int)lst.size();
    for (int q = 0; q < *n && q < cap; ++q) out[q] = L.neighbour_atom(atom, lst[q]);
    return ISING_OK;
}

extern "C" int ising_mesh_derivative_list(const ising_mesh* m, int64_t* out) {
    if (!m || !out) return fail(ISING_ERR_ARG, "NULL argument");
    const Lattice& L = m->lat;
    for (int64_t a = 0; a < L.natoms; ++a) {
        int ix, iy, iz, s;
        L.cell_of(a, &ix, &iy, &iz, &s);
        for (int d = 0; d < 6; ++d) out[a * 6 + d] = L.neighbour_atom(a, L.deriv[s * 6 + d]);
    }
    return ISING_OK;
}

extern "C" int ising_mesh_colouring(ising_mesh* m, const ising_params* p, int* colour_of, int* n_colours) {
    if (!m || !colour_of || !n_colours) return fail(ISING_ERR_ARG, "NULL argument");
    ISG_TRY(validate_params(p));
    const Lattice& L = m->lat;
    const bool sh2 = uses_shell2(L, *p);
    if (m->layout.cb == 1 && !sh2) {
        for (int64_t a = 0; a < L.natoms; ++a) {
            int ix, iy, iz, s;
            L.cell_of(a, &ix, &iy, &iz, &s);
            colour_of[a] = (ix + iy + iz) & 1;
        }
        *n_colours = 2;
        return ISING_OK;
    }
    Colouring& c = m->colour[sh2 ? 1 : 0];
    ISG_TRY(host_colouring(m, sh2, c));
    std::memcpy(colour_of, c.host_colour.data(), L.natoms * sizeof(int));
    *n_colours = c.ncol;
    return ISING_OK;
}

// ======================================================================= spins
namespace {
int staging(ising_mesh* m, double** d) {
    // FP64 staging for 3N doubles, allocated on first use
    const size_t need = (size_t)3 * m->lat.natoms;
    if (m->staging_size < need) {
        cudaFree(m->d_staging);
        m->d_staging = nullptr;
        m->staging_size = 0;
        ISG_TRY(dev_alloc(&m->d_staging, need));
        m->staging_size = need;
    }
    *d = m->d_staging;
    return ISING_OK;
}
}  // namespace

extern "C" int ising_spins_set(ising_mesh* m, int replica, const double* s) {
    ISG_TRY(check_replica(m, replica));
    if (!s) return fail(ISING_ERR_ARG, "spins array is NULL");
    DeviceGuard g(m->device);
    double* d;
    ISG_TRY(staging(m, &d));
    const int64_t N = m->lat.natoms;
    ISG_CUDA(cudaMemcpyAsync(d, s, (size_t)3 * N * sizeof(double), cudaMemcpyHostToDevice, m->stream));
    ISG_TRY(launch_spins_from_f64(d, m->d_spins + (int64_t)replica * 3 * N, N, m->layout, m->d_status, m->stream));
    return check_status(m);
}

extern "C" int ising_spins_get(const ising_mesh* mc, int replica, double* s) {
    ising_mesh* m = const_cast<ising_mesh*>(mc);
    ISG_TRY(check_replica(m, replica));
    if (!s) return fail(ISING_ERR_ARG, "spins array is NULL");
    DeviceGuard g(m->device);
    double* d;
    ISG_TRY(staging(m, &d));
    const int64_t N = m->lat.natoms;
    ISG_TRY(launch_spins_to_f64(m->d_spins + (int64_t)replica * 3 * N, d, N, m->layout, m->stream));
    ISG_CUDA(cudaMemcpyAsync(s, d, (size_t)3 * N * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    ISG_CUDA(cudaStreamSynchronize(m->stream));
    return ISING_OK;
}

namespace {

// Asynchronous transfers of a mesh: downloads on one stream, uploads on another, one FP64
// staging buffer per replica and, per replica, the events that order a download and an
// upload of the same replica (they share the staging buffer and, typically, the host array).
struct Xfer {
    cudaStream_t d2h = nullptr, h2d = nullptr;
    cudaEvent_t main_ready = nullptr;        // the mesh stream's work issued before a transfer
    std::vector<double*> stage;
    std::vector<cudaEvent_t> got, put;       // download / upload of replica r complete
    bool pending = false;
};

void xfer_release(ising_mesh* m) {
    Xfer* x = static_cast<Xfer*>(m->xfer);
    if (!x) return;
    if (x->d2h) { cudaStreamSynchronize(x->d2h); cudaStreamDestroy(x->d2h); }
    if (x->h2d) { cudaStreamSynchronize(x->h2d); cudaStreamDestroy(x->h2d); }
    if (x->main_ready) cudaEventDestroy(x->main_ready);
    for (double* d : x->stage) cudaFree(d);
    for (cudaEvent_t e : x->got) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : x->put) if (e) cudaEventDestroy(e);
    delete x;
    m->xfer = nullptr;
}

int xfer_state(ising_mesh* m, Xfer** out) {
    if (!m->xfer) {
        std::unique_ptr<Xfer> x(new Xfer());
        const int R = m->n_replicas;
        x->stage.assign(R, nullptr);
        x->got.assign(R, nullptr);
        x->put.assign(R, nullptr);
        m->xfer = x.release();
        Xfer* y = static_cast<Xfer*>(m->xfer);
        auto bail = [&](cudaError_t e, const char* what) { xfer_release(m); return cuda_fail(e, what); };
        cudaError_t e;
        if ((e = cudaStreamCreateWithFlags(&y->d2h, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
        if ((e = cudaStreamCreateWithFlags(&y->h2d, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
        if ((e = cudaEventCreateWithFlags(&y->main_ready, cudaEventDisableTiming)) != cudaSuccess) return bail(e, "event");
        for (int r = 0; r < R; ++r)
            if ((e = cudaEventCreateWithFlags(&y->got[r], cudaEventDisableTiming)) != cudaSuccess ||
                (e = cudaEventCreateWithFlags(&y->put[r], cudaEventDisableTiming)) != cudaSuccess)
                return bail(e, "event");
    }
    *out = static_cast<Xfer*>(m->xfer);
    return ISING_OK;
}

}  // namespace

int isg::mesh_settle(const ising_mesh* mc) {
    ising_mesh* m = const_cast<ising_mesh*>(mc);
    Xfer* x = m ? static_cast<Xfer*>(m->xfer) : nullptr;
    if (!x || !x->pending) return ISING_OK;
    DeviceGuard g(m->device);
    x->pending = false;
    ISG_CUDA(cudaStreamSynchronize(x->d2h));
    ISG_CUDA(cudaStreamSynchronize(x->h2d));
    return check_status(m);   // an upload of non-finite or zero spins set the status word
}

extern "C" int ising_spins_get_async(ising_mesh* m, int replica, double* s) {
    ISG_TRY(check_replica_only(m, replica));
    if (!s) return fail(ISING_ERR_ARG, "spins array is NULL");
    DeviceGuard g(m->device);
    Xfer* x;
    ISG_TRY(xfer_state(m, &x));
    const int64_t N = m->lat.natoms;
    if (!x->stage[replica]) ISG_TRY(dev_alloc(&x->stage[replica], (size_t)3 * N));
    // after the work already issued on the mesh's stream and any upload of this replica
    ISG_CUDA(cudaEventRecord(x->main_ready, m->stream));
    ISG_CUDA(cudaStreamWaitEvent(x->d2h, x->main_ready, 0));
    ISG_CUDA(cudaStreamWaitEvent(x->d2h, x->put[replica], 0));
    x->pending = true;
    ISG_TRY(launch_spins_to_f64(m->d_spins + (int64_t)replica * 3 * N, x->stage[replica], N, m->layout, x->d2h));
    ISG_CUDA(cudaMemcpyAsync(s, x->stage[replica], (size_t)3 * N * sizeof(double), cudaMemcpyDeviceToHost, x->d2h));
    ISG_CUDA(cudaEventRecord(x->got[replica], x->d2h));
    return ISING_OK;
}

extern "C" int ising_spins_set_async(ising_mesh* m, int replica, const double* s) {
    ISG_TRY(check_replica_only(m, replica));
    if (!s) return fail(ISING_ERR_ARG, "spins array is NULL");
    DeviceGuard g(m->device);
    Xfer* x;
    ISG_TRY(xfer_state(m, &x));
    const int64_t N = m->lat.natoms;
    if (!x->stage[replica]) ISG_TRY(dev_alloc(&x->stage[replica], (size_t)3 * N));
    // after the work already issued on the mesh's stream and any download of this replica
    // (which reads the same staging buffer and may fill the host array read here)
    ISG_CUDA(cudaEventRecord(x->main_ready, m->stream));
    ISG_CUDA(cudaStreamWaitEvent(x->h2d, x->main_ready, 0));
    ISG_CUDA(cudaStreamWaitEvent(x->h2d, x->got[replica], 0));
    x->pending = true;
    ISG_CUDA(cudaMemcpyAsync(x->stage[replica], s, (size_t)3 * N * sizeof(double), cudaMemcpyHostToDevice, x->h2d));
    ISG_TRY(launch_spins_from_f64(x->stage[replica], m->d_spins + (int64_t)replica * 3 * N, N, m->layout, m->d_status,
                                  x->h2d));
    ISG_CUDA(cudaEventRecord(x->put[replica], x->h2d));
    return ISING_OK;
}

extern "C" int ising_spins_wait(ising_mesh* m) {
    if (!m) return fail(ISING_ERR_ARG, "mesh is NULL");
    return mesh_settle(m);
}

extern "C" int ising_spins_init_uniform(ising_mesh* m, uint64_t seed, uint32_t ensemble) {
    ISG_TRY(check_replica(m, 0));
    if (ensemble >= (1u << 24)) return fail(ISING_ERR_ARG, "ensemble id must be < 2^24");
    DeviceGuard g(m->device);
    ISG_TRY(launch_init_uniform(m->d_spins, m->lat.natoms, m->layout, m->n_replicas, seed, ensemble, m->stream));
    ISG_CUDA(cudaStreamSynchronize(m->stream));
    return ISING_OK;
}

// ======================================================================= params
extern "C" int ising_params_reference(int which, double J, double Jp, double Dz, double Dzp, double B,
                                      ising_params* p) {
    if (!p) return fail(ISING_ERR_ARG, "params is NULL");
    std::memset(p, 0, sizeof *p);
    p->J = J; p->J_prime = Jp; p->Dz = Dz; p->Dz_prime = Dzp; p->B = B;
    p->K_axis[2] = 1.0;
    p->dmi_mode = ISING_DMI_INTERFACIAL;
    if (which == 0) {           // calculateHeisenbergEnergy / Metropolis_mcs
        p->zeeman_factor = 1.0;
        p->include_Jp = 1;
    } else if (which == 1) {    // TotalHeisenbergEnergy
        p->zeeman_factor = 2.0; // g * mu_B (src/constants.f90:11,14)
        p->include_Jp = 0;
        p->dmi_axis[2] = 1.0;   // [0, 0, Dz] (src/energyMin.f90:198)
        p->legacy_neighbours = 1;
    } else {
        return fail(ISING_ERR_ARG, "which must be 0 or 1");
    }
    return ISING_OK;
}

// ======================================================================= energies
extern "C" int ising_local_energy_batch(const ising_mesh* mc, int replica, int n, const int64_t* atoms,
                                        const double* sprop, const ising_params* p, double* old_e, double* new_e) {
    ising_mesh* m = const_cast<ising_mesh*>(mc);
    ISG_TRY(check_replica(m, replica));
    ISG_TRY(validate_params(p));
    if (n < 0 || (n > 0 && (!atoms || !sprop || !old_e || !new_e))) return fail(ISING_ERR_ARG, "bad batch arguments");
    for (int i = 0; i < n; ++i) {
        if (atoms[i] < 0 || atoms[i] >= m->lat.natoms) return fail(ISING_ERR_BOUNDS, "atom index out of range");
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(sprop[3 * i + k])) return fail(ISING_ERR_NAN, "NaN in proposed spin");
    }
    if (n == 0) return ISING_OK;
    DeviceGuard g(m->device);
    // scratch layout: atoms (n int64 as doubles), sprop (3n), old (n), new (n)
    const int chunk = kScratchDoubles / 6;
    ISG_TRY(upload_query_stencil(m, *p, false));
    if (p->demag) ISG_TRY(demag_enqueue(m, replica, true, false));
    for (int off = 0; off < n; off += chunk) {
        const int k = std::min(chunk, n - off);
        int64_t* d_atoms = reinterpret_cast<int64_t*>(m->d_scratch);
        double* d_sp = m->d_scratch + k;
        double* d_old = d_sp + 3 * k;
        double* d_new = d_old + k;
        std::memcpy(m->h_pinned, atoms + off, k * sizeof(int64_t));
        std::memcpy(m->h_pinned + k, sprop + 3 * off, 3 * k * sizeof(double));
        ISG_CUDA(cudaMemcpyAsync(m->d_scratch, m->h_pinned, 4 * k * sizeof(double), cudaMemcpyHostToDevice, m->stream));
        LocalLaunch a{};
        a.spins = m->d_spins + (int64_t)replica * 3 * m->lat.natoms;
        a.natoms = m->lat.natoms; a.nx = m->lat.nx; a.ny = m->lat.ny; a.nz = m->lat.nz; a.nsub = m->lat.nsub;
        a.ham = make_ham(*p); a.st = stencil_of(m); a.layout = m->layout; a.atoms = d_atoms; a.sprop = d_sp; a.old_e = d_old; a.new_e = d_new; a.n = k;
        a.demag_H = p->demag ? demag_field64(m) : nullptr;
        ISG_TRY(launch_local_energy(a, m->stream));
        ISG_CUDA(cudaMemcpyAsync(m->h_pinned + 4 * k, d_old, 2 * k * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
        ISG_CUDA(cudaStreamSynchronize(m->stream));
        std::memcpy(old_e + off, m->h_pinned + 4 * k, k * sizeof(double));
        std::memcpy(new_e + off, m->h_pinned + 5 * k, k * sizeof(double));
    }
    return ISING_OK;
}

extern "C" int ising_local_energy(const ising_mesh* m, int replica, int atom_1based, const ising_params* p,
                                  const double s_prop[3], double* old_e, double* new_e) {
    if (!m) return fail(ISING_ERR_ARG, "mesh is NULL");
    if (!s_prop || !old_e || !new_e) return fail(ISING_ERR_ARG, "NULL argument");
    if (atom_1based < 1 || atom_1based > m->lat.natoms) return fail(ISING_ERR_BOUNDS, "atomIndex out of range");
    const int64_t a = atom_1based - 1;
    return ising_local_energy_batch(m, replica, 1, &a, s_prop, p, old_e, new_e);
}

extern "C" int ising_observables(const ising_mesh* mc, const ising_params* p, double* e, double* mv) {
    ising_mesh* m = const_cast<ising_mesh*>(mc);
    ISG_TRY(check_replica(m, 0));
    ISG_TRY(validate_params(p));
    DeviceGuard g(m->device);
    const int R = m->n_replicas;
    const int tmp = energy_tmp_doubles(m, R);
    double* d_tmp = nullptr;
    ISG_TRY(dev_alloc(&d_tmp, (size_t)tmp + 4 * R));
    int st = enqueue_energy(m, *p, 0, R, d_tmp + tmp, d_tmp);
    std::vector<double> h(4 * R);
    if (st == ISING_OK) {
        cudaError_t ce = cudaMemcpyAsync(h.data(), d_tmp + tmp, 4 * R * sizeof(double), cudaMemcpyDeviceToHost, m->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(m->stream);
        if (ce != cudaSuccess) st = cuda_fail(ce, "observables copy");
    }
    cudaFree(d_tmp);
    if (st != ISING_OK) return st;
    if (p->demag)   // -1/2 mu_0 S.H with the field of the current spins (src/energyMin.f90:223-226, 511)
        for (int r = 0; r < R; ++r) {
            double dot = 0.0;
            ISG_TRY(demag_enqueue(m, r, true, false));
            ISG_TRY(demag_dot(m, r, &dot));
            h[4 * r] += -0.5 * kMu0 * dot;
        }
    for (int r = 0; r < R; ++r) {
        if (e) e[r] = h[4 * r];
        if (mv) for (int k = 0; k < 3; ++k) mv[3 * r + k] = h[4 * r + 1 + k];
    }
    return ISING_OK;
}

extern "C" int ising_total_energy(const ising_mesh* mc, int replica, const ising_params* p, double* e) {
    ising_mesh* m = const_cast<ising_mesh*>(mc);
    ISG_TRY(check_replica(m, replica));
    ISG_TRY(validate_params(p));
    if (!e) return fail(ISING_ERR_ARG, "e is NULL");
    DeviceGuard g(m->device);
    const int tmp = energy_tmp_doubles(m, 1);
    double* d_tmp = nullptr;
    ISG_TRY(dev_alloc(&d_tmp, (size_t)tmp + 4));
    int st = enqueue_energy(m, *p, replica, 1, d_tmp + tmp, d_tmp);
    double h[4] = {0, 0, 0, 0};
    if (st == ISING_OK) {
        cudaError_t ce = cudaMemcpyAsync(h, d_tmp + tmp, 4 * sizeof(double), cudaMemcpyDeviceToHost, m->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(m->stream);
        if (ce != cudaSuccess) st = cuda_fail(ce, "energy copy");
    }
    cudaFree(d_tmp);
    if (st != ISING_OK) return st;
    if (p->demag) {   // -1/2 mu_0 S.H with the field of the current spins (src/energyMin.f90:223-226, 511)
        double dot = 0.0;
        ISG_TRY(demag_enqueue(m, replica, true, false));
        ISG_TRY(demag_dot(m, replica, &dot));
        h[0] += -0.5 * kMu0 * dot;
    }
    *e = h[0];
    return ISING_OK;
}

extern "C" int ising_demag_field(const ising_mesh* mc, int replica, double* H) {
    ising_mesh* m = const_cast<ising_mesh*>(mc);
    ISG_TRY(check_replica(m, replica));
    if (!H) return fail(ISING_ERR_ARG, "H is NULL");
    DeviceGuard g(m->device);
    ISG_TRY(mesh_settle(m));
    ISG_TRY(demag_enqueue(m, replica, true, false));
    ISG_CUDA(cudaMemcpyAsync(H, demag_field64(m), 3 * (size_t)m->lat.natoms * sizeof(double), cudaMemcpyDeviceToHost,
                             m->stream));
    ISG_CUDA(cudaStreamSynchronize(m->stream));
    return ISING_OK;
}

// ======================================================================= sweeps
extern "C" int ising_metropolis_mcs(ising_mesh* m, int replica, double beta, int n_sweeps, const ising_params* p,
                                    double r, uint64_t seed) {
    ISG_TRY(check_replica(m, replica));
    ISG_TRY(validate_params(p));
    if (n_sweeps < 0) return fail(ISING_ERR_ARG, "numMCSSweeps must be >= 0");
    if (!std::isfinite(beta) || !std::isfinite(r)) return fail(ISING_ERR_NAN, "non-finite beta or r");
    if (n_sweeps == 0) return ISING_OK;
    DeviceGuard g(m->device);
    SweepPlan plan;
    ISG_TRY(make_plan(m, *p, &plan, m->d_slots, m->d_slot_count));
    const int move = r > 0.0 ? 1 : 0;
    m->h_pinned[0] = beta;
    ISG_CUDA(cudaMemcpyAsync(m->d_beta + replica, m->h_pinned, sizeof(double), cudaMemcpyHostToDevice, m->stream));
    if (p->demag) {
        // the field is computed at the start and after every demag_update_interval =
        // int(pi sqrt(5) / (2 r)) sweeps (src/energyMin.f90:258-259, 363-366); the uniform move
        // (r <= 0) keeps the field of the start
        const double pi_f = (double)3.14159265358979323846f;
        const int every = move ? std::max(1, (int)(pi_f * std::sqrt(5.0) / (2.0 * r))) : n_sweeps;
        plan.demag = demag_field32(m);
        for (int sw0 = 0; sw0 < n_sweeps; sw0 += every) {
            ISG_TRY(demag_enqueue(m, replica, false, true));
            plan.demag = demag_field32(m);
            ISG_TRY(enqueue_sweeps(m, plan, replica, 1, m->d_beta, (uint32_t)sw0, std::min(every, n_sweeps - sw0), seed,
                                   0u, move, r, nullptr));
        }
    } else {
        ISG_TRY(enqueue_sweeps(m, plan, replica, 1, m->d_beta, 0u, n_sweeps, seed, 0u, move, r, nullptr));
    }
    ISG_TRY(launch_advance(m->d_sweep + replica, 1, (uint32_t)n_sweeps, m->stream));
    m->h_sweep[replica] += (uint32_t)n_sweeps;
    return check_status(m);
}

// ======================================================================= winding
extern "C" int ising_winding_all_slices(const ising_mesh* mc, int replica, double* q) {
    ising_mesh* m = const_cast<ising_mesh*>(mc);
    ISG_TRY(check_replica(m, replica));
    if (!q) return fail(ISING_ERR_ARG, "q is NULL");
    DeviceGuard g(m->device);
    const Lattice& L = m->lat;
    WindingLaunch w{};
    w.spins = m->d_spins + (int64_t)replica * 3 * L.natoms;
    w.natoms = L.natoms; w.nx = L.nx; w.ny = L.ny; w.nz = L.nz; w.nsub = L.nsub; w.n_rep = 1;
    w.plaq = m->d_plaq; w.layout = m->layout; w.out = m->d_winding_tmp; w.fp64 = 1;
    ISG_TRY(launch_winding(w, m->stream));
    ISG_CUDA(cudaMemcpyAsync(q, m->d_winding_tmp, L.nz * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    ISG_CUDA(cudaStreamSynchronize(m->stream));
    return ISING_OK;
}

extern "C" int ising_winding_number(const ising_mesh* m, int replica, int z1, double* q) {
    if (!m) return fail(ISING_ERR_ARG, "mesh is NULL");
    if (z1 < 1 || z1 > m->lat.nz) return fail(ISING_ERR_BOUNDS, "Z_index out of bounds");
    if (!q) return fail(ISING_ERR_ARG, "q is NULL");
    std::vector<double> all(m->lat.nz);
    ISG_TRY(ising_winding_all_slices(m, replica, all.data()));
    *q = all[z1 - 1];
    return ISING_OK;
}

extern "C" int ising_statistics(const ising_mesh* m, int replica, double* wnd_mid, double* wnd_spread, double mv[3]) {
    ISG_TRY(check_replica(m, replica));
    if (m->lat.nz < 2) return fail(ISING_ERR_BOUNDS, "numCellsZ/2 is 0");
    std::vector<double> all(m->lat.nz);
    ISG_TRY(ising_winding_all_slices(m, replica, all.data()));
    const double mx = *std::max_element(all.begin(), all.end());
    const double mn = *std::min_element(all.begin(), all.end());
    if (wnd_spread) *wnd_spread = std::fabs(mx - mn);
    if (wnd_mid) *wnd_mid = all[m->lat.nz / 2 - 1];
    if (mv) {
        ising_params p{};
        p.zeeman_factor = 1.0;
        std::vector<double> e(m->n_replicas), mm(3 * m->n_replicas);
        ISG_TRY(ising_observables(m, &p, e.data(), mm.data()));
        for (int k = 0; k < 3; ++k) mv[k] = mm[3 * replica + k] / (double)m->lat.natoms;
    }
    return ISING_OK;
}

// plaquette densities (rsp:438-500) of slices z0 .. z0+nzc-1 from k_winding in FP64, written
// column-major per slice (x fastest) into the staging buffer (cells <= atoms < 3N doubles) and
// downloaded once
namespace {
int winding_density_range(const ising_mesh* mc, int replica, int z0, int nzc, double* dens) {
    ising_mesh* m = const_cast<ising_mesh*>(mc);
    ISG_TRY(check_replica(m, replica));
    if (!dens) return fail(ISING_ERR_ARG, "density is NULL");
    DeviceGuard g(m->device);
    const Lattice& L = m->lat;
    double* d = nullptr;
    ISG_TRY(staging(m, &d));
    WindingLaunch w{};
    w.spins = m->d_spins + (int64_t)replica * 3 * L.natoms;
    w.natoms = L.natoms; w.nx = L.nx; w.ny = L.ny; w.nz = L.nz; w.nsub = L.nsub; w.n_rep = 1;
    w.plaq = m->d_plaq; w.layout = m->layout; w.out = m->d_winding_tmp; w.fp64 = 1;
    w.dens = d; w.z0 = z0; w.nzc = nzc;
    ISG_TRY(launch_winding(w, m->stream));
    const size_t n = (size_t)L.nx * L.ny * nzc;
    ISG_CUDA(cudaMemcpyAsync(dens, d, n * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    ISG_CUDA(cudaStreamSynchronize(m->stream));
    return ISING_OK;
}
}  // namespace

extern "C" int ising_winding_density(const ising_mesh* m, int replica, int z1, double* dens) {
    if (!m) return fail(ISING_ERR_ARG, "mesh is NULL");
    if (z1 < 1 || z1 > m->lat.nz) return fail(ISING_ERR_BOUNDS, "Z_index out of bounds");
    return winding_density_range(m, replica, z1 - 1, 1, dens);
}

extern "C" int ising_winding_density_all(const ising_mesh* m, int replica, double* dens) {
    if (!m) return fail(ISING_ERR_ARG, "mesh is NULL");
    return winding_density_range(m, replica, 0, m->lat.nz, dens);
}

// ======================================================================= parallel tempering
struct ising_pt {
    ising_mesh* mesh = nullptr;
    int n = 0;
    ising_params p{};
    ising_pt_options opt{};
    SweepPlan plan;
    double* d_beta_t = nullptr;
    double* d_beta_rep = nullptr;
    int* d_t2r = nullptr;
    int* d_r2t = nullptr;
    Acc4* d_acc = nullptr;
    double* d_partials = nullptr;
    unsigned long long* d_stats = nullptr;
    uint32_t* d_round = nullptr;
    double* d_series = nullptr;
    int* d_count = nullptr;
    double* d_q = nullptr;
    double* d_energy_tmp = nullptr;
    double* d_energy_out = nullptr;
    Slot* d_plan_slots = nullptr;
    int* d_plan_count = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_k = -1;
    int rounds_done = 0;
    // learned patch move workspace (allocated by the first patch call)
    float *pw_win = nullptr, *pw_winp = nullptr, *pw_prop = nullptr;
    double *pw_lqf = nullptr, *pw_dE = nullptr, *pw_dM = nullptr;
    int *pw_rej = nullptr, *pw_acc = nullptr;
    unsigned long long* pw_stats = nullptr;
    float* pw_scale = nullptr;          // per-slot step scale (null: 1)
    double* pw_jump = nullptr;          // per-slot sum of squared spin displacements of accepted patches
    float pw_drift = 1.f;               // weight of the network's mean rotation
    int pw_batch = 0;
    int64_t pw_windows = 0;
    uint32_t patch_round = 0;
};

namespace {
void pt_free(ising_pt* pt) {
    if (pt->graph) cudaGraphExecDestroy(pt->graph);
    cudaFree(pt->d_beta_t); cudaFree(pt->d_beta_rep); cudaFree(pt->d_t2r); cudaFree(pt->d_r2t);
    cudaFree(pt->d_acc); cudaFree(pt->d_partials); cudaFree(pt->d_stats); cudaFree(pt->d_round);
    cudaFree(pt->d_series); cudaFree(pt->d_count); cudaFree(pt->d_q); cudaFree(pt->d_energy_tmp);
    cudaFree(pt->d_energy_out); cudaFree(pt->d_plan_slots); cudaFree(pt->d_plan_count);
    cudaFree(pt->pw_win); cudaFree(pt->pw_winp); cudaFree(pt->pw_prop); cudaFree(pt->pw_lqf); cudaFree(pt->pw_dE);
    cudaFree(pt->pw_dM); cudaFree(pt->pw_rej); cudaFree(pt->pw_acc); cudaFree(pt->pw_stats); cudaFree(pt->pw_scale);
    cudaFree(pt->pw_jump);
}

int pt_resync_enqueue(ising_pt* pt) {
    ising_mesh* m = pt->mesh;
    ISG_TRY(mesh_settle(m));
    ISG_TRY(enqueue_energy(m, pt->p, 0, pt->n, pt->d_energy_out, pt->d_energy_tmp));
    ISG_CUDA(cudaMemcpyAsync(pt->d_acc, pt->d_energy_out, (size_t)pt->n * 4 * sizeof(double),
                             cudaMemcpyDeviceToDevice, m->stream));
    return ISING_OK;
}

// Enqueue one PT round: k sweeps of replicas 0..n-1 (recording after each sweep when asked),
// fold the per-block partial sums into the FP64 accumulators, exchange, advance counters.
int pt_enqueue_round(ising_pt* pt, int k) {
    ising_mesh* m = pt->mesh;
    ISG_TRY(mesh_settle(m));
    const int n = pt->n;
    const int move = pt->opt.move;
    if (!pt->opt.record)
        ISG_TRY(enqueue_sweeps(m, pt->plan, 0, n, pt->d_beta_rep, 0u, k, pt->opt.seed, pt->opt.ensemble, move,
                               pt->opt.r, pt->d_partials));
    for (int sw = 0; sw < k && pt->opt.record; ++sw) {
        ISG_TRY(enqueue_sweep(m, pt->plan, 0, n, pt->d_beta_rep, (uint32_t)sw, pt->opt.seed, pt->opt.ensemble, move,
                              pt->opt.r, pt->d_partials));
        {
            ISG_TRY(launch_fold_partials(pt->d_partials, pt->plan.slots_per_rep, n, pt->d_acc, m->stream));
            // FP64, as the reference computes arc_winding: in FP32 a nearly antiparallel
            // neighbour pair rounds 1 + s_i.s_j to <= 0, and the normalisation sqrt of the
            // Berg-Luscher term is NaN (seen in hot replicas every few hundred sweeps)
            WindingLaunch w{};
            w.spins = m->d_spins; w.natoms = m->lat.natoms; w.nx = m->lat.nx; w.ny = m->lat.ny; w.nz = m->lat.nz;
            w.nsub = m->lat.nsub; w.n_rep = n; w.plaq = m->d_plaq; w.layout = m->layout; w.out = pt->d_q; w.fp64 = 1;
            ISG_TRY(launch_winding(w, m->stream));
            RecordLaunch rl{};
            rl.acc = pt->d_acc; rl.q = pt->d_q; rl.t2r = pt->d_t2r; rl.nz = m->lat.nz; rl.n_rep = n;
            rl.natoms = m->lat.natoms; rl.series = pt->d_series; rl.cap = pt->opt.record_capacity; rl.count = pt->d_count;
            ISG_TRY(launch_record(rl, m->stream));
        }
    }
    if (!pt->opt.record)
        ISG_TRY(launch_fold_partials(pt->d_partials, pt->plan.slots_per_rep, n, pt->d_acc, m->stream));
    ExchangeLaunch ex{};
    ex.n = n; ex.beta_t = pt->d_beta_t; ex.beta_rep = pt->d_beta_rep; ex.t2r = pt->d_t2r; ex.r2t = pt->d_r2t;
    ex.acc = pt->d_acc; ex.stats = pt->d_stats; ex.round = pt->d_round; ex.seed = pt->opt.seed;
    ex.ensemble = pt->opt.ensemble; ex.scheme = pt->opt.scheme;
    ISG_TRY(launch_exchange(ex, m->stream));
    ISG_TRY(launch_advance(m->d_sweep, n, (uint32_t)k, m->stream));
    return ISING_OK;
}
}  // namespace

extern "C" int ising_pt_create(ising_mesh* m, int n, const double* betas, const ising_params* p,
                               const ising_pt_options* opt, ising_pt** out) {
    if (!out) return fail(ISING_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!m || !betas || !opt) return fail(ISING_ERR_ARG, "NULL argument");
    ISG_TRY(mesh_settle(m));
    ISG_TRY(check_replica(m, 0));
    ISG_TRY(validate_params(p));
    if (p->demag)   // the reference's drivers run with demag = .false. (src/PT.f90:29, src/ISING.f90:46)
        return fail(ISING_ERR_UNSUPPORTED, "parallel tempering runs without the demagnetising field");
    if (n < 1 || n > m->n_replicas) return fail(ISING_ERR_ARG, "n_temps must be in 1..n_replicas");
    for (int t = 0; t < n; ++t) if (!std::isfinite(betas[t])) return fail(ISING_ERR_NAN, "non-finite beta");
    if (opt->move != ISING_MOVE_UNIFORM && opt->move != ISING_MOVE_BALL) return fail(ISING_ERR_ARG, "bad move");
    if (opt->scheme != ISING_PT_EVEN_ODD && opt->scheme != ISING_PT_RANDOM_PAIRS) return fail(ISING_ERR_ARG, "bad scheme");
    if (opt->ensemble >= (1u << 24)) return fail(ISING_ERR_ARG, "ensemble id must be < 2^24");
    if (opt->record && opt->record_capacity < 1) return fail(ISING_ERR_ARG, "record_capacity must be >= 1");
    DeviceGuard g(m->device);
    std::unique_ptr<ising_pt> pt(new ising_pt());
    pt->mesh = m; pt->n = n; pt->p = *p; pt->opt = *opt;
    auto bail = [&](int s) { pt_free(pt.get()); return s; };
    int st = ISING_OK;
    if ((st = dev_alloc(&pt->d_plan_slots, (size_t)kMaxSub * kMaxSlots)) ||
        (st = dev_alloc(&pt->d_plan_count, kMaxSub)))
        return bail(st);
    if ((st = make_plan(m, *p, &pt->plan, pt->d_plan_slots, pt->d_plan_count)) != ISING_OK) return bail(st);
    if (opt->l2_group < 0) return bail(fail(ISING_ERR_ARG, "l2_group must be >= 0"));
    if (opt->l2_group > 0) pt->plan.group = opt->l2_group;
    if (opt->sweep_kernel < 0 || opt->sweep_kernel > 3) return bail(fail(ISING_ERR_ARG, "sweep_kernel must be 0..3"));
    if (opt->sweep_kernel == 3) {   // octant meshes: every sweep of a round in one persistent launch
        if (m->layout.cb != 2 || pt->plan.oct_maxcnt < 1)
            return bail(fail(ISING_ERR_ARG, "the persistent octant engine needs an octant-layout mesh"));
        pt->plan.oct_engine = true;
    }
    if (opt->sweep_kernel == 2) {
        const Lattice& Lt = m->lat;
        if (!pt->plan.sc || !cb_tma_supported(Lt.nx, Lt.ny, Lt.nz))
            return bail(fail(ISING_ERR_ARG, "the TMA-staged kernel needs a checkerboard mesh with nz % 8 == 0"));
        pt->plan.tma = true;
        pt->plan.slots_per_rep = std::max(pt->plan.slots_per_rep, cb_tma_slots_per_rep(Lt.nx, Lt.ny, Lt.nz));
    }
    const int tmp = energy_tmp_doubles(m, n);
    if ((st = dev_alloc(&pt->d_beta_t, n)) || (st = dev_alloc(&pt->d_beta_rep, m->n_replicas)) ||
        (st = dev_alloc(&pt->d_t2r, n)) || (st = dev_alloc(&pt->d_r2t, n)) || (st = dev_alloc(&pt->d_acc, n)) ||
        (st = dev_alloc(&pt->d_partials, (size_t)n * pt->plan.slots_per_rep * 4)) ||
        (st = dev_alloc(&pt->d_stats, 2 * (size_t)n)) || (st = dev_alloc(&pt->d_round, 1)) ||
        (st = dev_alloc(&pt->d_count, 1)) || (st = dev_alloc(&pt->d_q, (size_t)n * m->lat.nz)) ||
        (st = dev_alloc(&pt->d_energy_tmp, tmp)) || (st = dev_alloc(&pt->d_energy_out, 4 * (size_t)n)))
        return bail(st);
    if (opt->record && (st = dev_alloc(&pt->d_series, (size_t)n * opt->record_capacity * 4))) return bail(st);
    std::vector<int> ident(n);
    for (int t = 0; t < n; ++t) ident[t] = t;
    cudaError_t ce = cudaMemcpy(pt->d_beta_t, betas, n * sizeof(double), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemcpy(pt->d_beta_rep, betas, n * sizeof(double), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemcpy(pt->d_t2r, ident.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemcpy(pt->d_r2t, ident.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemset(pt->d_partials, 0, (size_t)n * pt->plan.slots_per_rep * 4 * sizeof(double));
    if (ce == cudaSuccess) ce = cudaMemset(pt->d_stats, 0, 2 * (size_t)n * sizeof(unsigned long long));
    if (ce == cudaSuccess) ce = cudaMemset(pt->d_round, 0, sizeof(uint32_t));
    if (ce == cudaSuccess) ce = cudaMemset(pt->d_count, 0, sizeof(int));
    if (ce != cudaSuccess) return bail(cuda_fail(ce, "pt init"));
    if ((st = pt_resync_enqueue(pt.get())) != ISING_OK) return bail(st);
    if ((ce = cudaStreamSynchronize(m->stream)) != cudaSuccess) return bail(cuda_fail(ce, "pt init sync"));
    *out = pt.release();
    return ISING_OK;
}

extern "C" int ising_pt_destroy(ising_pt* pt) {
    if (!pt) return ISING_OK;
    DeviceGuard g(pt->mesh->device);
    cudaStreamSynchronize(pt->mesh->stream);
    pt_free(pt);
    delete pt;
    return ISING_OK;
}

extern "C" int ising_pt_run(ising_pt* pt, int k, int rounds) {
    if (!pt) return fail(ISING_ERR_ARG, "pt is NULL");
    if (k < 1 || rounds < 0) return fail(ISING_ERR_ARG, "sweeps_per_swap must be >= 1 and rounds >= 0");
    ising_mesh* m = pt->mesh;
    ISG_TRY(mesh_settle(m));
    DeviceGuard g(m->device);
    if (pt->graph_k != k) {
        if (pt->graph) { cudaGraphExecDestroy(pt->graph); pt->graph = nullptr; }
        cudaGraph_t graph;
        ISG_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
        int st = pt_enqueue_round(pt, k);
        cudaError_t ce = cudaStreamEndCapture(m->stream, &graph);
        if (st != ISING_OK) { if (ce == cudaSuccess) cudaGraphDestroy(graph); return st; }
        ISG_CUDA(ce);
        ce = cudaGraphInstantiate(&pt->graph, graph, 0);
        cudaGraphDestroy(graph);
        ISG_CUDA(ce);
        pt->graph_k = k;
    }
    for (int r = 0; r < rounds; ++r) {
        ISG_CUDA(cudaGraphLaunch(pt->graph, m->stream));
        ++pt->rounds_done;
        if (pt->opt.resync_every > 0 && pt->rounds_done % pt->opt.resync_every == 0) ISG_TRY(pt_resync_enqueue(pt));
    }
    if (pt->plan.oct_stall) {   // an injected stall lasts one call: capture the plain round again
        ISG_CUDA(cudaStreamSynchronize(m->stream));
        pt->plan.oct_stall = 0;
        pt->plan.oct_wait_ns = 2000000000ull;
        if (pt->graph) { cudaGraphExecDestroy(pt->graph); pt->graph = nullptr; }
        pt->graph_k = -1;
    }
    return check_status(m);
}

extern "C" int ising_pt_inject_stall(ising_pt* pt, int wait_ms) {
    if (!pt) return fail(ISING_ERR_ARG, "pt is NULL");
    if (!pt->plan.oct_engine) return fail(ISING_ERR_ARG, "stall injection needs the persistent octant engine");
    if (wait_ms < 1 || wait_ms > 60000) return fail(ISING_ERR_ARG, "wait_ms must be 1..60000");
    DeviceGuard g(pt->mesh->device);
    ISG_CUDA(cudaStreamSynchronize(pt->mesh->stream));
    pt->plan.oct_stall = 1;
    pt->plan.oct_wait_ns = (uint64_t)wait_ms * 1000000ull;
    if (pt->graph) { cudaGraphExecDestroy(pt->graph); pt->graph = nullptr; }
    pt->graph_k = -1;
    return ISING_OK;
}

extern "C" int ising_pt_relax(ising_pt* pt, int n_sweeps) {
    if (!pt) return fail(ISING_ERR_ARG, "pt is NULL");
    if (n_sweeps < 0) return fail(ISING_ERR_ARG, "n_sweeps must be >= 0");
    ising_mesh* m = pt->mesh;
    ISG_TRY(mesh_settle(m));
    DeviceGuard g(m->device);
    ISG_TRY(enqueue_sweeps(m, pt->plan, 0, pt->n, pt->d_beta_rep, 0u, n_sweeps, pt->opt.seed, pt->opt.ensemble,
                           pt->opt.move, pt->opt.r, pt->d_partials));
    ISG_TRY(launch_fold_partials(pt->d_partials, pt->plan.slots_per_rep, pt->n, pt->d_acc, m->stream));
    ISG_TRY(launch_advance(m->d_sweep, pt->n, (uint32_t)n_sweeps, m->stream));
    return check_status(m);
}

extern "C" int ising_pt_schedule(const ising_pt* pt, int k, int* group, int* launches, int* kernel) {
    if (!pt) return fail(ISING_ERR_ARG, "pt is NULL");
    if (k < 1) return fail(ISING_ERR_ARG, "sweeps_per_swap must be >= 1");
    const SweepPlan& P = pt->plan;
    const bool oct = !P.sc && pt->mesh->layout.cb == 2;
    int grp = (P.sc || oct) ? std::min(P.group, pt->n) : pt->n;
    int G = (pt->n + grp - 1) / grp;
    int L = 0;
    if (P.sc) L = G > 1 ? G * k + 1 : 2 * k;
    else if (P.bip) { L = 2 * k; grp = pt->n; }
    else if (oct && P.oct_engine) { L = 1; grp = pt->n; }
    else if (oct) {
        for (const auto& c : P.col->oct_blocks) L += octant_class_launches((int)c.size(), P.oct_maxcnt);
        L *= G * k;
    }
    else L = k * P.col->ncol;
    if (group) *group = grp;
    if (launches) *launches = L;
    // 0 k_general_colour / k_octant_colour, 1 k_cb_sweep, 2 k_cb_tma, 3 k_octant_fast,
    // 4 k_octant_engine, 5 k_bip_sweep, 6 k_octant_pair
    const int fast = pt->mesh->lat.nz % 4 == 0 ? 6 : 3;
    if (kernel)
        *kernel = P.sc ? (P.tma ? 2 : 1) : P.bip ? 5 : (oct ? (P.oct_engine ? 4 : (P.oct_maxcnt > 0 ? fast : 0)) : 0);
    return ISING_OK;
}

extern "C" int ising_pt_permutation(const ising_pt* pt, int* t2r) {
    if (!pt || !t2r) return fail(ISING_ERR_ARG, "NULL argument");
    DeviceGuard g(pt->mesh->device);
    ISG_CUDA(cudaMemcpyAsync(t2r, pt->d_t2r, pt->n * sizeof(int), cudaMemcpyDeviceToHost, pt->mesh->stream));
    ISG_CUDA(cudaStreamSynchronize(pt->mesh->stream));
    return ISING_OK;
}

extern "C" int ising_pt_energies(const ising_pt* pt, double* e, double* mv) {
    if (!pt) return fail(ISING_ERR_ARG, "pt is NULL");
    DeviceGuard g(pt->mesh->device);
    std::vector<Acc4> h(pt->n);
    ISG_CUDA(cudaMemcpyAsync(h.data(), pt->d_acc, pt->n * sizeof(Acc4), cudaMemcpyDeviceToHost, pt->mesh->stream));
    ISG_CUDA(cudaStreamSynchronize(pt->mesh->stream));
    for (int r = 0; r < pt->n; ++r) {
        if (e) e[r] = h[r].e;
        if (mv) { mv[3 * r] = h[r].mx; mv[3 * r + 1] = h[r].my; mv[3 * r + 2] = h[r].mz; }
    }
    return ISING_OK;
}

extern "C" int ising_pt_resync(ising_pt* pt) {
    if (!pt) return fail(ISING_ERR_ARG, "pt is NULL");
    DeviceGuard g(pt->mesh->device);
    ISG_TRY(pt_resync_enqueue(pt));
    ISG_CUDA(cudaStreamSynchronize(pt->mesh->stream));
    return ISING_OK;
}

extern "C" int ising_pt_swap_stats(const ising_pt* pt, uint64_t* att, uint64_t* acc) {
    if (!pt) return fail(ISING_ERR_ARG, "pt is NULL");
    DeviceGuard g(pt->mesh->device);
    std::vector<unsigned long long> h(2 * (size_t)pt->n);
    ISG_CUDA(cudaMemcpyAsync(h.data(), pt->d_stats, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             pt->mesh->stream));
    ISG_CUDA(cudaStreamSynchronize(pt->mesh->stream));
    for (int t = 0; t + 1 < pt->n; ++t) {
        if (att) att[t] = h[t];
        if (acc) acc[t] = h[(pt->n - 1) + t];
    }
    return ISING_OK;
}

extern "C" int ising_pt_series(const ising_pt* pt, double* out, int* n_rec) {
    if (!pt || !n_rec) return fail(ISING_ERR_ARG, "NULL argument");
    if (!pt->opt.record) return fail(ISING_ERR_ARG, "recording was not enabled");
    DeviceGuard g(pt->mesh->device);
    int c = 0;
    ISG_CUDA(cudaMemcpyAsync(&c, pt->d_count, sizeof(int), cudaMemcpyDeviceToHost, pt->mesh->stream));
    ISG_CUDA(cudaStreamSynchronize(pt->mesh->stream));
    *n_rec = c;
    if (out)
        ISG_CUDA(cudaMemcpy(out, pt->d_series, (size_t)pt->n * pt->opt.record_capacity * 4 * sizeof(double),
                            cudaMemcpyDeviceToHost));
    return ISING_OK;
}

// ======================================================================= helpers for noalloc.cu

// ======================================================================= learned patch move
namespace {

int patch_setup(ising_pt* pt, int colour, int offx, int offy, int offz, int slots, PatchStep* P, int* n_slots) {
    ising_mesh* m = pt->mesh;
    ISG_TRY(mesh_settle(m));
    const Lattice& L = m->lat;
    if (!pt->plan.sc || L.nsub != 1) return fail(ISING_ERR_UNSUPPORTED, "the patch move needs a simple-cubic mesh with shell-1 couplings");
    if (L.nx % 8 || L.ny % 8 || L.nz % 8) return fail(ISING_ERR_ARG, "the patch move needs nx, ny, nz divisible by 8");
    if (colour < 0 || colour > 7) return fail(ISING_ERR_ARG, "colour must be 0..7");
    if (offx < 0 || offx > 7 || offy < 0 || offy > 7 || offz < 0 || offz > 7) return fail(ISING_ERR_ARG, "offsets must be 0..7");
    if (slots < 0 || slots > pt->n) return fail(ISING_ERR_ARG, "slots must be 0..n_temps");
    *n_slots = slots ? slots : pt->n;
    PatchStep& Q = *P;
    Q = PatchStep{};
    Q.spins = m->d_spins; Q.natoms = L.natoms; Q.nx = L.nx; Q.ny = L.ny; Q.nz = L.nz; Q.layout = m->layout;
    Q.colour = colour; Q.offx = offx; Q.offy = offy; Q.offz = offz;
    Q.per_slot = (L.nx / 8) * (L.ny / 8) * (L.nz / 8);
    Q.t2r = pt->d_t2r; Q.beta_rep = pt->d_beta_rep; Q.ham = pt->plan.ham; Q.step_scale = pt->pw_scale; Q.drift = pt->pw_drift;
    Q.seed = pt->opt.seed; Q.ensemble = pt->opt.ensemble; Q.status = m->d_status;
    return ISING_OK;
}

int patch_workspace(ising_pt* pt, int batch) {
    ising_mesh* m = pt->mesh;
    ISG_TRY(mesh_settle(m));
    const int64_t windows = (int64_t)pt->n * (m->lat.nx / 8) * (m->lat.ny / 8) * (m->lat.nz / 8);
    if (pt->pw_batch >= batch && pt->pw_windows >= windows) return ISING_OK;
    cudaFree(pt->pw_win); cudaFree(pt->pw_winp); cudaFree(pt->pw_prop); cudaFree(pt->pw_lqf); cudaFree(pt->pw_dE);
    cudaFree(pt->pw_dM); cudaFree(pt->pw_rej); cudaFree(pt->pw_acc);
    pt->pw_win = pt->pw_winp = pt->pw_prop = nullptr;
    pt->pw_lqf = pt->pw_dE = pt->pw_dM = nullptr;
    pt->pw_rej = pt->pw_acc = nullptr;
    pt->pw_batch = 0;
    pt->pw_windows = 0;
    ISG_TRY(dev_alloc(&pt->pw_win, (size_t)batch * 1536));
    ISG_TRY(dev_alloc(&pt->pw_winp, (size_t)batch * 1536));
    ISG_TRY(dev_alloc(&pt->pw_prop, (size_t)batch * 192));
    ISG_TRY(dev_alloc(&pt->pw_lqf, batch));
    ISG_TRY(dev_alloc(&pt->pw_rej, batch));
    ISG_TRY(dev_alloc(&pt->pw_dE, windows));
    ISG_TRY(dev_alloc(&pt->pw_dM, 4 * windows));
    ISG_TRY(dev_alloc(&pt->pw_acc, windows));
    if (!pt->pw_stats) {
        ISG_TRY(dev_alloc(&pt->pw_stats, 2 * (size_t)pt->n));
        ISG_CUDA(cudaMemset(pt->pw_stats, 0, 2 * (size_t)pt->n * sizeof(unsigned long long)));
        ISG_TRY(dev_alloc(&pt->pw_jump, pt->n));
        ISG_CUDA(cudaMemset(pt->pw_jump, 0, (size_t)pt->n * sizeof(double)));
    }
    pt->pw_batch = batch;
    pt->pw_windows = windows;
    return ISING_OK;
}

}  // namespace

extern "C" int ising_pt_patch_set_scale(ising_pt* pt, const float* scale_per_slot, float drift) {
    if (!pt) return fail(ISING_ERR_ARG, "pt is NULL");
    if (!(drift >= 0.f) || !std::isfinite(drift)) return fail(ISING_ERR_ARG, "drift must be >= 0");
    DeviceGuard g(pt->mesh->device);
    pt->pw_drift = drift;
    if (!scale_per_slot) {
        cudaFree(pt->pw_scale);
        pt->pw_scale = nullptr;
        return ISING_OK;
    }
    for (int t = 0; t < pt->n; ++t)
        if (!(scale_per_slot[t] > 0.f) || !std::isfinite(scale_per_slot[t])) return fail(ISING_ERR_ARG, "step scales must be positive");
    if (!pt->pw_scale) ISG_TRY(dev_alloc(&pt->pw_scale, pt->n));
    ISG_CUDA(cudaMemcpyAsync(pt->pw_scale, scale_per_slot, pt->n * sizeof(float), cudaMemcpyHostToDevice, pt->mesh->stream));
    ISG_CUDA(cudaStreamSynchronize(pt->mesh->stream));
    return ISING_OK;
}

extern "C" int ising_pt_patch_count(const ising_pt* pt, int slots, int64_t* n_windows) {
    if (!pt || !n_windows) return fail(ISING_ERR_ARG, "NULL argument");
    const Lattice& L = pt->mesh->lat;
    if (slots < 0 || slots > pt->n) return fail(ISING_ERR_ARG, "slots must be 0..n_temps");
    *n_windows = (int64_t)(slots ? slots : pt->n) * (L.nx / 8) * (L.ny / 8) * (L.nz / 8);
    return ISING_OK;
}

extern "C" int ising_pt_patch_step(ising_pt* pt, ising_net* net, int colour, int offx, int offy, int offz, int slots) {
    if (!pt || !net) return fail(ISING_ERR_ARG, "NULL argument");
    ising_mesh* m = pt->mesh;
    ISG_TRY(mesh_settle(m));
    if (net_device(net) != m->device) return fail(ISING_ERR_ARG, "network and mesh are on different devices");
    DeviceGuard g(m->device);
    PatchStep P;
    int ns = 0;
    ISG_TRY(patch_setup(pt, colour, offx, offy, offz, slots, &P, &ns));
    const int batch = net_max_batch(net);
    ISG_TRY(patch_workspace(pt, batch));
    P.round = pt->patch_round++;
    const int64_t total = (int64_t)ns * P.per_slot;
    cudaStream_t s = m->stream;
    for (int64_t w0 = 0; w0 < total; w0 += batch) {
        const int nb = (int)std::min<int64_t>(batch, total - w0);
        const float* out = nullptr;
        ISG_TRY(launch_patch_gather(P, w0, nb, nullptr, pt->pw_win, s, net_rows(net)));
        ISG_TRY(net_forward_prepared(net, nb, s, &out));
        ISG_TRY(launch_patch_propose(P, w0, nb, pt->pw_win, out, pt->pw_prop, pt->pw_lqf, pt->pw_rej, s));
        ISG_TRY(launch_patch_gather(P, w0, nb, pt->pw_prop, pt->pw_winp, s, net_rows(net)));
        ISG_TRY(net_forward_prepared(net, nb, s, &out));
        ISG_TRY(launch_patch_accept(P, w0, nb, pt->pw_win, pt->pw_winp, out, pt->pw_prop, pt->pw_lqf, pt->pw_rej,
                                    pt->pw_dE, pt->pw_dM, pt->pw_acc, s));
    }
    ISG_TRY(launch_patch_fold(P, ns, total, pt->pw_dE, pt->pw_dM, pt->pw_acc, pt->d_acc, pt->pw_stats, pt->pw_jump, s));
    ISG_TRY(net_status_on(net, s));
    return check_status(m);
}

extern "C" int ising_pt_patch_samples(ising_pt* pt, int colour, int offx, int offy, int offz, int slots, int n_local,
                                      float* d_windows, float* d_targets) {
    if (!pt || !d_windows || !d_targets) return fail(ISING_ERR_ARG, "NULL argument");
    if (n_local < 0) return fail(ISING_ERR_ARG, "n_local must be >= 0");
    ising_mesh* m = pt->mesh;
    ISG_TRY(mesh_settle(m));
    DeviceGuard g(m->device);
    PatchStep P;
    int ns = 0;
    ISG_TRY(patch_setup(pt, colour, offx, offy, offz, slots, &P, &ns));
    P.round = pt->patch_round++;
    const int64_t total = (int64_t)ns * P.per_slot;
    const int chunk = 1 << 16;
    for (int64_t w0 = 0; w0 < total; w0 += chunk) {
        const int nb = (int)std::min<int64_t>(chunk, total - w0);
        ISG_TRY(launch_patch_gather(P, w0, nb, nullptr, d_windows + w0 * 1536, m->stream));
        ISG_TRY(launch_patch_equilibrate(P, w0, nb, d_windows + w0 * 1536, n_local, pt->opt.move, (float)pt->opt.r,
                                         d_targets + w0 * 192, m->stream));
    }
    return check_status(m);
}

extern "C" int ising_pt_patch_last(const ising_pt* pt, int n, float* win, float* winp, double* lqf, double* dE,
                                   int* accepted) {
    if (!pt) return fail(ISING_ERR_ARG, "pt is NULL");
    if (n < 0 || n > pt->pw_batch || n > pt->pw_windows) return fail(ISING_ERR_ARG, "n exceeds the last patch batch");
    DeviceGuard g(pt->mesh->device);
    cudaStream_t s = pt->mesh->stream;
    if (win) ISG_CUDA(cudaMemcpyAsync(win, pt->pw_win, (size_t)n * 1536 * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (winp) ISG_CUDA(cudaMemcpyAsync(winp, pt->pw_winp, (size_t)n * 1536 * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (lqf) ISG_CUDA(cudaMemcpyAsync(lqf, pt->pw_lqf, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (dE) ISG_CUDA(cudaMemcpyAsync(dE, pt->pw_dE, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (accepted) ISG_CUDA(cudaMemcpyAsync(accepted, pt->pw_acc, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, s));
    ISG_CUDA(cudaStreamSynchronize(s));
    return ISING_OK;
}

extern "C" int ising_pt_patch_jump(const ising_pt* pt, double* sq_jump) {
    if (!pt || !sq_jump) return fail(ISING_ERR_ARG, "NULL argument");
    DeviceGuard g(pt->mesh->device);
    for (int t = 0; t < pt->n; ++t) sq_jump[t] = 0.0;
    if (pt->pw_jump) {
        ISG_CUDA(cudaMemcpyAsync(sq_jump, pt->pw_jump, pt->n * sizeof(double), cudaMemcpyDeviceToHost, pt->mesh->stream));
        ISG_CUDA(cudaStreamSynchronize(pt->mesh->stream));
    }
    return ISING_OK;
}

extern "C" int ising_pt_patch_stats(const ising_pt* pt, uint64_t* proposed, uint64_t* accepted) {
    if (!pt) return fail(ISING_ERR_ARG, "pt is NULL");
    DeviceGuard g(pt->mesh->device);
    std::vector<unsigned long long> h(2 * (size_t)pt->n, 0ull);
    if (pt->pw_stats) {
        ISG_CUDA(cudaMemcpyAsync(h.data(), pt->pw_stats, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 pt->mesh->stream));
        ISG_CUDA(cudaStreamSynchronize(pt->mesh->stream));
    }
    for (int t = 0; t < pt->n; ++t) {
        if (proposed) proposed[t] = h[2 * t];
        if (accepted) accepted[t] = h[2 * t + 1];
    }
    return ISING_OK;
}

// ======================================================================= batched ensembles
namespace {

struct EnsHost {
    ising_mesh* mesh = nullptr;
    int n = 0;
    ising_params p{};
    uint32_t ensemble = 0;
    HamDev ham{};
    int dmi_kind = 0;
    double* d_beta_t = nullptr;
    double* d_beta_rep = nullptr;
    int* d_t2r = nullptr;
    int* d_r2t = nullptr;
    Acc4* d_acc = nullptr;
    unsigned long long* d_stats = nullptr;
    uint32_t* d_round = nullptr;
    double* d_energy_tmp = nullptr;
    double* d_energy_out = nullptr;
    uint32_t P = 1, nch = 1;        // x-planes per chunk, tasks per replica and colour pass (sweep when fused)
    size_t part_off = 0, done_off = 0;
    float* d_spins_b = nullptr;     // fused loader: second spin buffer of replicas 0..n-1
    uint32_t fnch = 1, fnseg = 1, fnp = 0;   // fused loader: chunks, y-segments, thread rows per block
};

// sync words, zeroed before every launch: head, abort, where, (pad), ready[kMaxEnsembles],
// fin[kMaxEnsembles] (64-bit), then the done counters of every replica's chunks
constexpr size_t kSyncReady = 4;
constexpr size_t kSyncFin = kSyncReady + kMaxEnsembles;   // word offset, 8-byte aligned
constexpr size_t kSyncDone = kSyncFin + 2 * kMaxEnsembles;

}  // namespace

struct ising_ensembles {
    std::vector<EnsHost> ens;
    ising_ensembles_options opt{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;   // the engine's own stream (never a mesh's)
    int move = 1, dmi = 0;
    bool has_k = false;
    ising_ensembles_schedule_t sched{256, 4096, ISING_ENS_ORDER_PHASE, 48000000, 0.0};
    int grid = 0;
    size_t fu_smem = 0;             // fused loader: dynamic shared memory per block
    std::vector<uint2> table;
    int table_k = -1;
    uint2* d_table = nullptr;
    size_t table_cap = 0;
    double* d_partials = nullptr;
    size_t partials_cap = 0;
    uint32_t* d_sync = nullptr;
    size_t sync_cap = 0, sync_words = 0;
    int* d_status = nullptr;
    uint32_t* h_words = nullptr;    // pinned: status, where
    cudaGraphExec_t graph = nullptr;
    int graph_k = -1, graph_rounds = -1;
    int64_t rounds_done = 0;
    int stall_next = -1;
};

namespace {

void ens_free(ising_ensembles* s) {
    if (s->graph) cudaGraphExecDestroy(s->graph);
    for (auto& h : s->ens) {
        cudaFree(h.d_beta_t); cudaFree(h.d_beta_rep); cudaFree(h.d_t2r); cudaFree(h.d_r2t); cudaFree(h.d_acc);
        cudaFree(h.d_stats); cudaFree(h.d_round); cudaFree(h.d_energy_tmp); cudaFree(h.d_energy_out);
        cudaFree(h.d_spins_b);
    }
    cudaFree(s->d_table); cudaFree(s->d_partials); cudaFree(s->d_sync); cudaFree(s->d_status);
    if (s->h_words) cudaFreeHost(s->h_words);
    if (s->own_stream) cudaStreamDestroy(s->own_stream);
}

void ens_drop_graph(ising_ensembles* s) {
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    s->graph_k = s->graph_rounds = -1;
}

// Every ensemble suits the staged loader: packed rows of 64 entries (nz = 128), whole groups
// of kStG x-planes, and the driver's tensor-map encoder is present.
bool ens_staged_fits(const ising_ensembles* s) {
    if (!tensor_map_encoder()) return false;
    for (const auto& h : s->ens) {
        const Lattice& L = h.mesh->lat;
        if (L.nz != 128 || L.nx % kStG != 0) return false;
    }
    return true;
}

// Chunking, grid and buffers for schedule `c`.
int ens_apply_schedule(ising_ensembles* s, const ising_ensembles_schedule_t& c) {
    const bool fused = c.loader == ISING_ENS_LOADER_FUSED;
    if (fused) {
        if (c.block_threads < 128 || c.block_threads > kFuMaxThreads || c.block_threads % 32)
            return fail(ISING_ERR_ARG, "the fused loader runs 128..512-thread blocks in whole warps");
    } else if (c.block_threads < 64 || c.block_threads > kEnsMaxThreads || c.block_threads % 32) {
        return fail(ISING_ERR_ARG, "block_threads must be 64..256 in whole warps");
    }
    if (c.chunk_pairs < 1) return fail(ISING_ERR_ARG, "chunk_pairs must be >= 1");
    if (c.order != ISING_ENS_ORDER_PHASE && c.order != ISING_ENS_ORDER_GROUPS && c.order != ISING_ENS_ORDER_WAVE)
        return fail(ISING_ERR_ARG, "order must be ISING_ENS_ORDER_PHASE, _GROUPS or _WAVE");
    if (c.order == ISING_ENS_ORDER_GROUPS && c.group_bytes < 1) return fail(ISING_ERR_ARG, "group_bytes must be >= 1");
    if (c.loader != ISING_ENS_LOADER_REGISTERS && c.loader != ISING_ENS_LOADER_STAGED && !fused)
        return fail(ISING_ERR_ARG, "loader must be ISING_ENS_LOADER_REGISTERS, _STAGED or _FUSED");
    if (fused && c.order != ISING_ENS_ORDER_PHASE) return fail(ISING_ERR_ARG, "the fused loader queues in phase order");
    const bool staged = c.loader == ISING_ENS_LOADER_STAGED;
    if (staged) {
        if (c.block_threads != kStSub * kStG * 32) return fail(ISING_ERR_ARG, "the staged loader runs 256-thread blocks");
        if (!ens_staged_fits(s)) return fail(ISING_ERR_ARG, "the staged loader needs nz = 128 and nx % 4 == 0 in every ensemble");
    }
    size_t part = 0, done = 0, fu_smem = 0;
    for (auto& h : s->ens) {
        const Lattice& L = h.mesh->lat;
        if (fused) {
            // one thread row per x-plane of a chunk plus two halo planes; chunks of at least
            // two planes and y-segments of at least two rows keep every task's reads inside
            // its 3 x 3 neighbourhood of units
            const uint32_t G = (uint32_t)L.nz / 4u, rows = (uint32_t)c.block_threads / G;
            if (rows < 4) return fail(ISING_ERR_ARG, "the fused loader needs block_threads >= nz of every ensemble");
            const uint32_t pm = std::min<uint32_t>(rows - 2u, (uint32_t)L.nx);
            const uint32_t nch = ((uint32_t)L.nx + pm - 1u) / pm;
            const uint32_t widest = ((uint32_t)L.nx + nch - 1u) / nch;
            const double yl = std::max(2.0, (double)c.chunk_pairs / ((double)widest * G));
            long nseg = std::lround((double)L.ny / yl);
            nseg = std::max(1L, std::min(nseg, (long)L.ny / 2));
            if ((uint64_t)nch * (uint64_t)nseg >= 65536u) return fail(ISING_ERR_ARG, "too many fused units per replica");
            h.fnch = nch;
            h.fnseg = (uint32_t)nseg;
            h.fnp = widest + 2u;
            h.P = widest;
            h.nch = nch * (uint32_t)nseg;
            fu_smem = std::max(fu_smem, (size_t)(3u * (h.fnp + 2u) + 3u * h.fnp) * 3u * ((uint32_t)L.nz / 2u) * 4u);
            h.part_off = part;
            h.done_off = done;
            part += (size_t)h.n * h.nch * 4;
            done += (size_t)h.n * h.nch;
            continue;
        }
        const int lanes = L.nz / 4;   // W / 2
        if (lanes > c.block_threads) return fail(ISING_ERR_ARG, "block_threads smaller than nz / 4 of an ensemble");
        const double plane_pairs = (double)L.ny * lanes;
        int P = (int)std::lround((double)c.chunk_pairs / plane_pairs);
        P = std::max(1, std::min(P, L.nx));
        if (staged) P = std::max(kStG, P / kStG * kStG);   // whole plane groups (nx % kStG == 0)
        h.P = (uint32_t)P;
        h.nch = (uint32_t)((L.nx + P - 1) / P);
        h.part_off = part;
        h.done_off = done;
        part += (size_t)h.n * h.nch * 4;
        done += (size_t)h.n * h.nch;
    }
    if (fu_smem > 227u * 1024u) return fail(ISING_ERR_ARG, "fused loader: rows of the chunk exceed shared memory");
    const int loader = fused ? 2 : (staged ? 1 : 0);
    int per_sm = 0;
    ISG_TRY(ensembles_blocks_per_sm(s->move, s->dmi, s->has_k, loader, c.block_threads, fu_smem, &per_sm));
    if (per_sm < 1) return fail(ISING_ERR_CUDA, "persistent engine kernel cannot be resident");
    int sms = 0;
    ISG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
    ISG_CUDA(cudaStreamSynchronize(s->stream));
    if (fused)
        for (auto& h : s->ens)
            if (!h.d_spins_b) ISG_TRY(dev_alloc(&h.d_spins_b, (size_t)3 * (size_t)h.mesh->lat.natoms * (size_t)h.n));
    s->fu_smem = fu_smem;
    if (part > s->partials_cap) {
        cudaFree(s->d_partials);
        s->d_partials = nullptr;
        s->partials_cap = 0;
        ISG_TRY(dev_alloc(&s->d_partials, part));
        s->partials_cap = part;
    }
    // partial sums are zero between rounds; a new layout starts from zero as well
    ISG_CUDA(cudaMemsetAsync(s->d_partials, 0, s->partials_cap * sizeof(double), s->stream));
    const size_t words = kSyncDone + done;
    if (words > s->sync_cap) {
        cudaFree(s->d_sync);
        s->d_sync = nullptr;
        s->sync_cap = 0;
        ISG_TRY(dev_alloc(&s->d_sync, words));
        s->sync_cap = words;
    }
    s->sync_words = words;
    s->grid = per_sm * sms;
    s->sched = c;
    s->sched.ms_per_round = 0.0;
    s->table_k = -1;
    ens_drop_graph(s);
    return ISING_OK;
}

// Task table of one round: groups of replicas (all replicas in PHASE order), each running
// its 2k colour passes in turn; within a pass, replica by replica, chunk by chunk.
int ens_build_table(ising_ensembles* s, int k) {
    if (s->table_k == k) return ISING_OK;
    struct Unit { int e, r; double bytes; };
    std::vector<Unit> units;
    for (int e = 0; e < (int)s->ens.size(); ++e)
        for (int r = 0; r < s->ens[e].n; ++r) units.push_back({e, r, 12.0 * (double)s->ens[e].mesh->lat.natoms});
    std::vector<std::pair<size_t, size_t>> groups;   // [begin, end) into units
    if (s->sched.order == ISING_ENS_ORDER_PHASE) {
        groups.push_back({0, units.size()});
    } else {
        size_t b = 0;
        double acc = 0.0;
        for (size_t i = 0; i < units.size(); ++i) {
            if (i > b && acc + units[i].bytes > (double)s->sched.group_bytes) {
                groups.push_back({b, i});
                b = i;
                acc = 0.0;
            }
            acc += units[i].bytes;
        }
        groups.push_back({b, units.size()});
    }
    s->table.clear();
    if (s->sched.loader == ISING_ENS_LOADER_FUSED) {
        // one task per (replica, sweep, unit), sweep by sweep: a task only waits for the
        // previous sweep
        for (int sw = 0; sw < k; ++sw)
            for (size_t u = 0; u < units.size(); ++u) {
                const EnsHost& h = s->ens[units[u].e];
                for (uint32_t ch = 0; ch < h.nch; ++ch)
                    s->table.push_back(make_uint2(((uint32_t)units[u].e << 24) | (uint32_t)units[u].r,
                                                  ((uint32_t)sw << 16) | ch));
            }
    } else if (s->sched.order == ISING_ENS_ORDER_WAVE) {
        // wave key 3 ph + ((ch - ph) mod nch): each task's dependencies (the previous pass on
        // chunks ch-1, ch, ch+1, cyclic) have strictly smaller keys, so ordering by key (ties
        // by replica, then chunk) keeps every task after the tasks it waits for
        struct Keyed { uint64_t key; uint2 task; };
        std::vector<Keyed> all;
        for (size_t u = 0; u < units.size(); ++u) {
            const EnsHost& h = s->ens[units[u].e];
            for (int ph = 0; ph < 2 * k; ++ph)
                for (uint32_t ch = 0; ch < h.nch; ++ch) {
                    const uint64_t w = 3ull * (uint64_t)ph + (uint64_t)((ch + h.nch - (uint32_t)ph % h.nch) % h.nch);
                    all.push_back({(w << 40) | ((uint64_t)u << 16) | ch,
                                   make_uint2(((uint32_t)units[u].e << 24) | (uint32_t)units[u].r,
                                              ((uint32_t)ph << 16) | ch)});
                }
        }
        std::sort(all.begin(), all.end(), [](const Keyed& a, const Keyed& b) { return a.key < b.key; });
        s->table.reserve(all.size());
        for (const auto& t : all) s->table.push_back(t.task);
    } else {
        for (const auto& g : groups)
            for (int ph = 0; ph < 2 * k; ++ph)
                for (size_t u = g.first; u < g.second; ++u) {
                    const EnsHost& h = s->ens[units[u].e];
                    for (uint32_t ch = 0; ch < h.nch; ++ch)
                        s->table.push_back(make_uint2(((uint32_t)units[u].e << 24) | (uint32_t)units[u].r,
                                                      ((uint32_t)ph << 16) | ch));
                }
    }
    if (s->table.size() >= (1u << 30)) return fail(ISING_ERR_ARG, "task table too large");
    ISG_CUDA(cudaStreamSynchronize(s->stream));
    if (s->table.size() > s->table_cap) {
        cudaFree(s->d_table);
        s->d_table = nullptr;
        s->table_cap = 0;
        ISG_TRY(dev_alloc(&s->d_table, s->table.size()));
        s->table_cap = s->table.size();
    }
    ISG_CUDA(cudaMemcpy(s->d_table, s->table.data(), s->table.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    s->table_k = k;
    ens_drop_graph(s);
    return ISING_OK;
}

void ens_params(const ising_ensembles* s, int k, int rounds, int stall, EnsParams* P) {
    std::memset(P, 0, sizeof(*P));
    for (size_t i = 0; i < s->ens.size(); ++i) {
        const EnsHost& h = s->ens[i];
        const Lattice& L = h.mesh->lat;
        EnsDev& d = P->e[i];
        d.g.ham = h.ham;
        d.g.nx = L.nx; d.g.ny = L.ny; d.g.nz = L.nz;
        d.g.W = (uint32_t)(L.nz / 2);
        d.g.half = (uint32_t)(L.natoms / 2);
        d.g.row_stride_x = d.g.W * (uint32_t)L.ny;
        d.g.ensemble = h.ensemble;
        d.g.r = (float)s->opt.r;
        d.spins = h.mesh->d_spins;
        d.N = (uint32_t)L.natoms;
        d.divNY = make_div((uint32_t)L.ny);
        d.divTX = make_div(d.g.W / 2u);
        d.P = h.P;
        d.nch = h.nch;
        d.rb = (uint32_t)s->sched.block_threads / (d.g.W / 2u);
        d.nseg = std::max(1u, std::min((uint32_t)L.ny, (d.rb + h.P - 1) / h.P));
        d.seg_len = ((uint32_t)L.ny + d.nseg - 1) / d.nseg;
        d.divSeg = make_div(d.nseg);
        if (s->sched.loader == ISING_ENS_LOADER_STAGED) {
            // units of a task (plane groups x y-segments) come in pairs, one per sub-block
            const uint32_t groups = h.P / (uint32_t)kStG;
            d.st_nseg = std::min<uint32_t>((uint32_t)L.ny, groups % 2 ? 2u : 1u);
            d.st_seg_len = ((uint32_t)L.ny + d.st_nseg - 1) / d.st_nseg;
        }
        if (s->sched.loader == ISING_ENS_LOADER_FUSED) {
            d.spins_b = h.d_spins_b;
            d.fnch = h.fnch;
            d.fnseg = h.fnseg;
            d.fnp = h.fnp;
        }
        d.n_rep = h.n;
        d.beta_rep = h.d_beta_rep;
        d.sweep_ctr = h.mesh->d_sweep;
        d.partials = s->d_partials + h.part_off;
        d.done = s->d_sync + kSyncDone + h.done_off;
        d.ready = s->d_sync + kSyncReady + i;
        d.fin = reinterpret_cast<unsigned long long*>(s->d_sync + kSyncFin) + i;
        d.acc = h.d_acc; d.beta_t = h.d_beta_t; d.t2r = h.d_t2r; d.r2t = h.d_r2t;
        d.stats = h.d_stats; d.round_ctr = h.d_round;
    }
    P->n_ens = (int)s->ens.size();
    P->table = s->d_table;
    P->tasks_per_round = (uint32_t)s->table.size();
    P->rounds = (uint32_t)rounds;
    P->k = (uint32_t)k;
    P->head = s->d_sync;
    P->abort = s->d_sync + 1;
    P->where = s->d_sync + 2;
    P->status = s->d_status;
    P->wait_ns = (uint64_t)(s->opt.wait_timeout_ms > 0 ? s->opt.wait_timeout_ms : 2000) * 1000000ull;
    P->scheme = s->opt.scheme;
    P->stall_ens = stall;
    P->seed = s->opt.seed;
    philox_round_keys(s->opt.seed, P->rk);
}

int ens_enqueue_launch(ising_ensembles* s, int k, int rounds, int stall) {
    EnsParams P;
    ens_params(s, k, rounds, stall, &P);
    const bool staged = s->sched.loader == ISING_ENS_LOADER_STAGED;
    if (staged)
        for (size_t i = 0; i < s->ens.size(); ++i) {
            const EnsHost& h = s->ens[i];
            const Lattice& L = h.mesh->lat;
            if (!ensembles_encode_maps(h.mesh->d_spins, L.nx, L.ny, h.n, &P.maps[i]))
                return fail(ISING_ERR_CUDA, "cuTensorMapEncodeTiled (staged loader) failed");
        }
    ISG_CUDA(cudaMemsetAsync(s->d_sync, 0, s->sync_words * sizeof(uint32_t), s->stream));
    const int loader = s->sched.loader == ISING_ENS_LOADER_FUSED ? 2 : (staged ? 1 : 0);
    return launch_ensembles(P, s->move, s->dmi, s->has_k, loader, s->sched.block_threads, s->grid, s->fu_smem,
                            s->stream);
}

int ens_resync_enqueue(ising_ensembles* s) {
    for (auto& h : s->ens) {
        ising_mesh* m = h.mesh;
        cudaStream_t keep = m->stream;
        m->stream = s->stream;
        const int st = enqueue_energy(m, h.p, 0, h.n, h.d_energy_out, h.d_energy_tmp);
        m->stream = keep;
        ISG_TRY(st);
        ISG_CUDA(cudaMemcpyAsync(h.d_acc, h.d_energy_out, (size_t)h.n * 4 * sizeof(double), cudaMemcpyDeviceToDevice,
                                 s->stream));
    }
    return ISING_OK;
}

// engine status -> error code; after a timeout the partial sums are cleared and the
// accumulators recomputed so that the engine stays usable
int ens_check(ising_ensembles* s) {
    ISG_CUDA(cudaMemcpyAsync(s->h_words, s->d_status, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    ISG_CUDA(cudaMemcpyAsync(s->h_words + 1, s->d_sync + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
    ISG_CUDA(cudaStreamSynchronize(s->stream));
    const int st = (int)s->h_words[0];
    if (!st) return ISING_OK;
    const uint32_t where = s->h_words[1];
    ISG_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream));
    if (st & kStatTimeout) {
        ISG_CUDA(cudaMemsetAsync(s->d_partials, 0, s->partials_cap * sizeof(double), s->stream));
        ISG_TRY(ens_resync_enqueue(s));
        ISG_CUDA(cudaStreamSynchronize(s->stream));
        char msg[160];
        std::snprintf(msg, sizeof msg, "device wait timed out at task %u of the round table", where ? where - 1 : 0u);
        return fail(ISING_ERR_TIMEOUT, msg);
    }
    if (st & kStatNan) return fail(ISING_ERR_NAN, "NaN in spins or proposals");
    return fail(ISING_ERR_BOUNDS, "device index out of bounds");
}

int ens_run(ising_ensembles* s, int k, int rounds) {
    // the fused loader alternates two buffers sweep by sweep: an even round ends in the mesh's own
    if (s->sched.loader == ISING_ENS_LOADER_FUSED && k % 2)
        return fail(ISING_ERR_ARG, "the fused loader needs an even number of sweeps per round");
    for (auto& h : s->ens) ISG_TRY(mesh_settle(h.mesh));   // the engine's stream reads the meshes' spins
    ISG_TRY(ens_build_table(s, k));
    const int64_t tpr = (int64_t)s->table.size();
    const int max_r = (int)std::max<int64_t>(1, ((int64_t)1 << 31) / std::max<int64_t>(tpr, 1) - 1);
    while (rounds > 0) {
        int R = std::min(rounds, max_r);
        if (s->opt.resync_every > 0)
            R = std::min<int64_t>(R, s->opt.resync_every - s->rounds_done % s->opt.resync_every);
        if (s->stall_next >= 0) {
            const int stall = s->stall_next;
            s->stall_next = -1;
            ISG_TRY(ens_enqueue_launch(s, k, R, stall));
        } else {
            if (!s->graph || s->graph_k != k || s->graph_rounds != R) {
                ens_drop_graph(s);
                cudaGraph_t g;
                ISG_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
                const int st = ens_enqueue_launch(s, k, R, -1);
                cudaError_t ce = cudaStreamEndCapture(s->stream, &g);
                if (st != ISING_OK) { if (ce == cudaSuccess) cudaGraphDestroy(g); return st; }
                ISG_CUDA(ce);
                ce = cudaGraphInstantiate(&s->graph, g, 0);
                cudaGraphDestroy(g);
                ISG_CUDA(ce);
                s->graph_k = k;
                s->graph_rounds = R;
            }
            ISG_CUDA(cudaGraphLaunch(s->graph, s->stream));
        }
        s->rounds_done += R;
        rounds -= R;
        if (s->opt.resync_every > 0 && s->rounds_done % s->opt.resync_every == 0) ISG_TRY(ens_resync_enqueue(s));
    }
    return ens_check(s);
}

int ens_index(const ising_ensembles* s, int e) {
    if (!s) return fail(ISING_ERR_ARG, "engine is NULL");
    if (e < 0 || e >= (int)s->ens.size()) return fail(ISING_ERR_BOUNDS, "ensemble index out of range");
    return ISING_OK;
}

}  // namespace

extern "C" int ising_ensembles_create(int n, const ising_ensemble_desc* desc, const ising_ensembles_options* opt,
                                      ising_ensembles** out) {
    if (!out) return fail(ISING_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!desc || !opt) return fail(ISING_ERR_ARG, "NULL argument");
    if (n < 1 || n > kMaxEnsembles) return fail(ISING_ERR_ARG, "n_ensembles must be 1..16");
    if (opt->move != ISING_MOVE_UNIFORM && opt->move != ISING_MOVE_BALL) return fail(ISING_ERR_ARG, "bad move");
    if (opt->scheme != ISING_PT_EVEN_ODD && opt->scheme != ISING_PT_RANDOM_PAIRS) return fail(ISING_ERR_ARG, "bad scheme");
    if (opt->resync_every < 0 || opt->wait_timeout_ms < 0) return fail(ISING_ERR_ARG, "negative option");
    if (!std::isfinite(opt->r)) return fail(ISING_ERR_NAN, "non-finite r");
    const int dev = desc[0].mesh ? desc[0].mesh->device : -1;
    std::vector<int> kinds;
    for (int e = 0; e < n; ++e) {
        const ising_ensemble_desc& d = desc[e];
        ISG_TRY(check_replica(d.mesh, 0));
        if (d.mesh->device != dev) return fail(ISING_ERR_ARG, "all meshes must be on one device");
        for (int f = 0; f < e; ++f)
            if (desc[f].mesh == d.mesh) return fail(ISING_ERR_ARG, "each ensemble needs its own mesh");
        ISG_TRY(validate_params(&d.params));
        if (d.params.demag) return fail(ISING_ERR_UNSUPPORTED, "the batched engine runs without the demagnetising field");
        const Lattice& L = d.mesh->lat;
        if (d.mesh->layout.cb != 1 || uses_shell2(L, d.params))
            return fail(ISING_ERR_UNSUPPORTED, "the batched engine needs colour-separated simple-cubic meshes "
                                               "(even nx, ny; nz % 4 == 0) and shell-1 couplings");
        if (L.nx > 65535 || L.natoms >= (int64_t)1 << 31) return fail(ISING_ERR_ARG, "mesh too large for the engine");
        if (d.n_temps < 1 || d.n_temps > d.mesh->n_replicas) return fail(ISING_ERR_ARG, "n_temps must be in 1..n_replicas");
        if (d.ensemble >= (1u << 24)) return fail(ISING_ERR_ARG, "ensemble id must be < 2^24");
        if (!d.betas) return fail(ISING_ERR_ARG, "betas is NULL");
        for (int t = 0; t < d.n_temps; ++t) if (!std::isfinite(d.betas[t])) return fail(ISING_ERR_NAN, "non-finite beta");
    }
    DeviceGuard g(dev);
    std::unique_ptr<ising_ensembles> s(new ising_ensembles());
    s->opt = *opt;
    s->device = dev;
    s->move = opt->move;
    auto bail = [&](int st) { ens_free(s.get()); return st; };
    int st = ISING_OK;
    if (cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(cuda_fail(cudaGetLastError(), "cudaStreamCreateWithFlags"));
    s->stream = s->own_stream;
    std::vector<int> dk;
    for (int e = 0; e < n; ++e) {
        const ising_ensemble_desc& d = desc[e];
        EnsHost h;
        h.mesh = d.mesh; h.n = d.n_temps; h.p = d.params; h.ensemble = d.ensemble;
        h.ham = make_ham(d.params);
        if ((st = sc_dmi(d.mesh, d.params, &h.ham, &h.dmi_kind)) != ISING_OK) return bail(st);
        if (h.ham.K != 0.f) s->has_k = true;
        dk.push_back(h.dmi_kind);
        s->ens.push_back(h);
    }
    // one kernel variant for all: the common DMI form, else the tabulated one (kind 0 is
    // kind 1 with D = 0)
    {
        int kind = 0;
        for (int k : dk) {
            if (k == 0) continue;
            if (kind == 0) kind = k;
            else if (kind != k) kind = 3;
        }
        s->dmi = kind;
    }
    for (int e = 0; e < n; ++e) {
        EnsHost& h = s->ens[e];
        ising_mesh* m = h.mesh;
        if ((st = cudaStreamSynchronize(m->stream)) != cudaSuccess) return bail(cuda_fail((cudaError_t)st, "mesh sync"));
        const int tmp = energy_tmp_doubles(m, h.n);
        if ((st = dev_alloc(&h.d_beta_t, h.n)) || (st = dev_alloc(&h.d_beta_rep, h.n)) ||
            (st = dev_alloc(&h.d_t2r, h.n)) || (st = dev_alloc(&h.d_r2t, h.n)) || (st = dev_alloc(&h.d_acc, h.n)) ||
            (st = dev_alloc(&h.d_stats, 2 * (size_t)h.n)) || (st = dev_alloc(&h.d_round, 1)) ||
            (st = dev_alloc(&h.d_energy_tmp, tmp)) || (st = dev_alloc(&h.d_energy_out, 4 * (size_t)h.n)))
            return bail(st);
        std::vector<int> ident(h.n);
        for (int t = 0; t < h.n; ++t) ident[t] = t;
        cudaError_t ce = cudaMemcpy(h.d_beta_t, desc[e].betas, h.n * sizeof(double), cudaMemcpyHostToDevice);
        if (ce == cudaSuccess) ce = cudaMemcpy(h.d_beta_rep, desc[e].betas, h.n * sizeof(double), cudaMemcpyHostToDevice);
        if (ce == cudaSuccess) ce = cudaMemcpy(h.d_t2r, ident.data(), h.n * sizeof(int), cudaMemcpyHostToDevice);
        if (ce == cudaSuccess) ce = cudaMemcpy(h.d_r2t, ident.data(), h.n * sizeof(int), cudaMemcpyHostToDevice);
        if (ce == cudaSuccess) ce = cudaMemset(h.d_stats, 0, 2 * (size_t)h.n * sizeof(unsigned long long));
        if (ce == cudaSuccess) ce = cudaMemset(h.d_round, 0, sizeof(uint32_t));
        if (ce != cudaSuccess) return bail(cuda_fail(ce, "ensemble init"));
    }
    if ((st = dev_alloc(&s->d_status, 1)) != ISING_OK) return bail(st);
    if (cudaMemset(s->d_status, 0, sizeof(int)) != cudaSuccess) return bail(cuda_fail(cudaGetLastError(), "status init"));
    if (cudaMallocHost((void**)&s->h_words, 4 * sizeof(uint32_t)) != cudaSuccess) {
        s->h_words = nullptr;
        return bail(fail(ISING_ERR_ALLOC, "cudaMallocHost failed"));
    }
    ising_ensembles_schedule_t c = s->sched;
    int max_lanes = 0;
    for (auto& h : s->ens) max_lanes = std::max(max_lanes, h.mesh->lat.nz / 4);
    if (max_lanes > c.block_threads) return bail(fail(ISING_ERR_ARG, "nz too large for the engine (nz <= 1024)"));
    if ((st = ens_apply_schedule(s.get(), c)) != ISING_OK) return bail(st);
    if ((st = ens_resync_enqueue(s.get())) != ISING_OK) return bail(st);
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) return bail(cuda_fail(cudaGetLastError(), "engine init sync"));
    *out = s.release();
    return ISING_OK;
}

extern "C" int ising_ensembles_destroy(ising_ensembles* s) {
    if (!s) return ISING_OK;
    DeviceGuard g(s->device);
    cudaStreamSynchronize(s->stream);
    ens_free(s);
    delete s;
    return ISING_OK;
}

extern "C" int ising_ensembles_set_stream(ising_ensembles* s, void* stream) {
    if (!s) return fail(ISING_ERR_ARG, "engine is NULL");
    DeviceGuard g(s->device);
    ISG_CUDA(cudaStreamSynchronize(s->stream));
    s->stream = stream ? static_cast<cudaStream_t>(stream) : s->own_stream;
    ens_drop_graph(s);
    return ISING_OK;
}

extern "C" int ising_ensembles_run(ising_ensembles* s, int k, int rounds) {
    if (!s) return fail(ISING_ERR_ARG, "engine is NULL");
    if (k < 1 || k > 32767 || rounds < 0) return fail(ISING_ERR_ARG, "sweeps_per_swap must be 1..32767 and rounds >= 0");
    DeviceGuard g(s->device);
    return ens_run(s, k, rounds);
}

extern "C" int ising_ensembles_set_schedule(ising_ensembles* s, const ising_ensembles_schedule_t* c) {
    if (!s || !c) return fail(ISING_ERR_ARG, "NULL argument");
    DeviceGuard g(s->device);
    return ens_apply_schedule(s, *c);
}

extern "C" int ising_ensembles_get_schedule(const ising_ensembles* s, ising_ensembles_schedule_t* c, int* grid,
                                            int64_t* tasks_per_pass) {
    if (!s) return fail(ISING_ERR_ARG, "engine is NULL");
    if (c) *c = s->sched;
    if (grid) *grid = s->grid;
    if (tasks_per_pass) {
        int64_t t = 0;
        for (const auto& h : s->ens) t += (int64_t)h.n * h.nch;
        *tasks_per_pass = t;
    }
    return ISING_OK;
}

extern "C" int ising_ensembles_autotune(ising_ensembles* s, int k, int rounds_per_trial,
                                        ising_ensembles_schedule_t* trials, int max_trials, int* n_trials) {
    if (!s) return fail(ISING_ERR_ARG, "engine is NULL");
    if (k < 1 || rounds_per_trial < 1) return fail(ISING_ERR_ARG, "sweeps_per_swap and rounds_per_trial must be >= 1");
    DeviceGuard g(s->device);
    std::vector<ising_ensembles_schedule_t> cand;
    int max_lanes = 0;
    for (auto& h : s->ens) max_lanes = std::max(max_lanes, h.mesh->lat.nz / 4);
    const int threads[] = {256, 128};
    const int chunks[] = {2048, 4096, 8192, 16384, 32768};
    for (int t : threads) {
        if (t < max_lanes) continue;
        for (int c : chunks) cand.push_back({t, c, ISING_ENS_ORDER_PHASE, 0, 0.0, ISING_ENS_LOADER_REGISTERS});
        // replica groups of ~64 MB (one L2-resident group per round); slower so far, kept as a candidate
        cand.push_back({t, 8192, ISING_ENS_ORDER_GROUPS, 64000000, 0.0, ISING_ENS_LOADER_REGISTERS});
    }
    // small meshes: tasks below one 2048-pair chunk keep enough of them per colour pass
    // (SC L=32 x 32 replicas: 512 pairs per task 5.3e10 updates/s against 3.4e10 at 2048)
    for (int c : {512, 1024}) cand.push_back({128, c, ISING_ENS_ORDER_PHASE, 0, 0.0, ISING_ENS_LOADER_REGISTERS});
    if (max_lanes <= 64)      // two-warp blocks (8 per SM, the same 16 warps) with small tasks
        for (int c : {2048, 4096}) cand.push_back({64, c, ISING_ENS_ORDER_PHASE, 0, 0.0, ISING_ENS_LOADER_REGISTERS});
    // rows of W/2 = 24 lanes (nz = 96, as in C5) leave 8 of 128 threads idle; 96-thread blocks
    // hold exactly four rows
    bool rows24 = true;
    for (auto& h : s->ens) rows24 = rows24 && h.mesh->lat.nz / 4 == 24;
    if (rows24)
        for (int c : {512, 1024, 2048, 4096}) cand.push_back({96, c, ISING_ENS_ORDER_PHASE, 0, 0.0, ISING_ENS_LOADER_REGISTERS});
    if (ens_staged_fits(s))   // groups of 4, 8 and 16 x-planes per task at nz = 128
        for (int c : {16384, 32768, 65536}) cand.push_back({256, c, ISING_ENS_ORDER_PHASE, 0, 0.0, ISING_ENS_LOADER_STAGED});
    if (k % 2 == 0)           // one pass per sweep: chunk widths by block size, y-segments by chunk_pairs
        for (int t : {256, 384, 480, 512})
            if (t >= 4 * max_lanes && (t != 480 || rows24))   // 480 = 20 whole rows of 24 lanes
                for (int c : {16384, 65536, 1 << 30})
                    cand.push_back({t, c, ISING_ENS_ORDER_PHASE, 0, 0.0, ISING_ENS_LOADER_FUSED});
    cudaEvent_t e0, e1;
    ISG_CUDA(cudaEventCreate(&e0));
    ISG_CUDA(cudaEventCreate(&e1));
    int best = -1, n = 0;
    int st = ISING_OK;
    for (size_t i = 0; i < cand.size() && st == ISING_OK; ++i) {
        if ((st = ens_apply_schedule(s, cand[i])) != ISING_OK) break;
        if ((st = ens_run(s, k, rounds_per_trial)) != ISING_OK) break;   // warm-up: table, graph
        cudaEventRecord(e0, s->stream);
        if ((st = ens_run(s, k, rounds_per_trial)) != ISING_OK) break;
        cudaEventRecord(e1, s->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        cand[i].ms_per_round = ms / rounds_per_trial;
        if (trials && n < max_trials) trials[n] = cand[i];
        ++n;
        if (best < 0 || cand[i].ms_per_round < cand[best].ms_per_round) best = (int)i;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (n_trials) *n_trials = n;
    if (st != ISING_OK) return st;
    if (best < 0) return fail(ISING_ERR_ARG, "no candidate schedule fits these ensembles");
    const double ms = cand[best].ms_per_round;
    ISG_TRY(ens_apply_schedule(s, cand[best]));
    s->sched.ms_per_round = ms;
    return ISING_OK;
}

extern "C" int ising_ensembles_permutation(const ising_ensembles* s, int e, int* t2r) {
    ISG_TRY(ens_index(s, e));
    if (!t2r) return fail(ISING_ERR_ARG, "NULL argument");
    DeviceGuard g(s->device);
    const EnsHost& h = s->ens[e];
    ISG_CUDA(cudaMemcpyAsync(t2r, h.d_t2r, h.n * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    ISG_CUDA(cudaStreamSynchronize(s->stream));
    return ISING_OK;
}

extern "C" int ising_ensembles_energies(const ising_ensembles* s, int e, double* E, double* M) {
    ISG_TRY(ens_index(s, e));
    DeviceGuard g(s->device);
    const EnsHost& h = s->ens[e];
    std::vector<Acc4> a(h.n);
    ISG_CUDA(cudaMemcpyAsync(a.data(), h.d_acc, h.n * sizeof(Acc4), cudaMemcpyDeviceToHost, s->stream));
    ISG_CUDA(cudaStreamSynchronize(s->stream));
    for (int r = 0; r < h.n; ++r) {
        if (E) E[r] = a[r].e;
        if (M) { M[3 * r] = a[r].mx; M[3 * r + 1] = a[r].my; M[3 * r + 2] = a[r].mz; }
    }
    return ISING_OK;
}

extern "C" int ising_ensembles_swap_stats(const ising_ensembles* s, int e, uint64_t* att, uint64_t* acc) {
    ISG_TRY(ens_index(s, e));
    DeviceGuard g(s->device);
    const EnsHost& h = s->ens[e];
    std::vector<unsigned long long> v(2 * (size_t)h.n);
    ISG_CUDA(cudaMemcpyAsync(v.data(), h.d_stats, v.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             s->stream));
    ISG_CUDA(cudaStreamSynchronize(s->stream));
    for (int t = 0; t + 1 < h.n; ++t) {
        if (att) att[t] = v[t];
        if (acc) acc[t] = v[(h.n - 1) + t];
    }
    return ISING_OK;
}

extern "C" int ising_ensembles_resync(ising_ensembles* s) {
    if (!s) return fail(ISING_ERR_ARG, "engine is NULL");
    DeviceGuard g(s->device);
    for (auto& h : s->ens) ISG_TRY(mesh_settle(h.mesh));
    ISG_TRY(ens_resync_enqueue(s));
    ISG_CUDA(cudaStreamSynchronize(s->stream));
    return ISING_OK;
}

extern "C" int ising_ensembles_set_resync(ising_ensembles* s, int every) {
    if (!s) return fail(ISING_ERR_ARG, "engine is NULL");
    if (every < 0) return fail(ISING_ERR_ARG, "resync interval must be >= 0");
    s->opt.resync_every = every;
    s->rounds_done = 0;
    return ISING_OK;
}

extern "C" int ising_ensembles_inject_stall(ising_ensembles* s, int e) {
    ISG_TRY(ens_index(s, e));
    s->stall_next = e;
    return ISING_OK;
}

namespace isg {
// Shell or legacy stencil of p written into caller-provided host memory (no allocation).
int fill_query_stencil_host(const ising_mesh* m, const ising_params& p, bool legacy, Slot* slots, int* cnt) {
    const Lattice& L = m->lat;
    for (int s = 0; s < kMaxSub; ++s) cnt[s] = 0;
    for (int s = 0; s < L.nsub; ++s) {
        int c = 0;
        auto add = [&](const NbrSlot& q, float w, bool dmi) -> int {
            if (c >= kMaxSlots) return fail(ISING_ERR_ARG, "stencil exceeds 128 slots");
            Slot e{};
            e.dx = (int8_t)q.dx; e.dy = (int8_t)q.dy; e.dz = (int8_t)q.dz; e.sub = (uint8_t)q.sub;
            e.w = w;
            if (dmi && p.Dz != 0.0) {
                double D[3];
                bond_dmi(L, p, q.r, D);
                e.Dx = (float)D[0]; e.Dy = (float)D[1]; e.Dz = (float)D[2];
            }
            slots[(size_t)s * kMaxSlots + c++] = e;
            return ISING_OK;
        };
        if (legacy) {
            for (const auto& q : L.legacy[s]) ISG_TRY(add(q, (float)p.J, true));
        } else {
            for (const auto& q : L.shell[0][s]) ISG_TRY(add(q, (float)p.J, true));
            if (uses_shell2(L, p))
                for (const auto& q : L.shell[1][s]) ISG_TRY(add(q, (float)p.J_prime, false));
        }
        cnt[s] = c;
    }
    return ISING_OK;
}
HamDev ham_of(const ising_params& p) { return make_ham(p); }
int check_params(const ising_params* p) { return validate_params(p); }
}  // namespace isg
