// Host orchestration of the B200 path: the mdelast_driver_* entry points of
// include/mdelast.h. A driver owns its device buffers and one stream; integrate() is one
// CUDA-graph launch per step (the two graphs differ in whether the step samples the Born
// tensor and the Laplacian). Results come back lazily: the graph's last node copies the
// scalar observables into pinned host memory and the first read after a step waits for it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "host_tables.h"
#include "gr_kernels.cuh"
#include "kernels.cuh"

using namespace mdelast;

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(MDELAST_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_),    \
                        __FILE__, __LINE__);                                                  \
    } while (0)

namespace {

// Device buffers come from a stream-ordered memory pool of this library's own, one per
// device, created on first use with a release threshold that keeps freed memory: a driver
// created after another was destroyed (the NPT and NVT stages of a protocol, a warm start's
// corrected boxes) reuses its pages instead of mapping new ones. The device's default pool,
// which other users in the process (PyTorch's cudaMallocAsync backend, for one) may tune
// for themselves, is left as it is. mdelast_release_cached_memory() trims this pool.
std::mutex g_pool_mutex;
std::vector<cudaMemPool_t> g_pools;

int own_pool(int dev, cudaMemPool_t *out) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (dev < 0)
        return fail(MDELAST_ERR_ARGUMENT, "device %d", dev);
    if (g_pools.size() <= static_cast<size_t>(dev))
        g_pools.resize(static_cast<size_t>(dev) + 1, nullptr);
    cudaMemPool_t &pool = g_pools[static_cast<size_t>(dev)];
    if (!pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        CK(cudaMemPoolCreate(&pool, &props));
        uint64_t keep = UINT64_MAX;
        CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    *out = pool;
    return MDELAST_OK;
}

// Allocated, zeroed and complete on return (the driver's own stream does not order against
// the legacy stream the pool is used on).
template <typename T> int dalloc(T **p, size_t n) {
    size_t const bytes = sizeof(T) * (n > 0 ? n : 1);
    int dev = 0;
    CK(cudaGetDevice(&dev));
    cudaMemPool_t pool = nullptr;
    if (int rc = own_pool(dev, &pool))
        return rc;
    CK(cudaMallocFromPoolAsync(reinterpret_cast<void **>(p), bytes, pool, cudaStreamLegacy));
    CK(cudaMemsetAsync(*p, 0, bytes, cudaStreamLegacy));
    CK(cudaStreamSynchronize(cudaStreamLegacy));
    return MDELAST_OK;
}

// Returned to the pool once all work on the device has finished, as cudaFree would wait.
template <typename T> void dfree(T *&p) {
    if (p) {
        cudaDeviceSynchronize();
        cudaFreeAsync(p, cudaStreamLegacy);
    }
    p = nullptr;
}

// Host staging of a creation's atom uploads: pinned, kept from one creation to the next (a
// batch created after another reuses it instead of faulting in and pinning fresh pages),
// used by one creation at a time under its mutex. mdelast_release_cached_memory() frees it.
std::mutex g_stage_mutex;
void *g_stage = nullptr;
size_t g_stage_bytes = 0;

// at least `bytes` of pinned staging (nullptr on failure); call with g_stage_mutex held
void *stage_host(size_t bytes) {
    if (bytes > g_stage_bytes) {
        if (g_stage)
            cudaFreeHost(g_stage);
        g_stage = nullptr;
        g_stage_bytes = 0;
        if (cudaHostAlloc(&g_stage, bytes, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            g_stage = nullptr;
            return nullptr;
        }
        g_stage_bytes = bytes;
    }
    return g_stage;
}

double nint_host(double x) { // md_driver.hpp:48-50
    return static_cast<double>(x < 0. ? static_cast<int>(x - 0.5) : static_cast<int>(x + 0.5));
}

// Lanes per atom for the pair passes: the fewest that give about 150k threads (enough to
// cover 148 SMs with the warps the register budget allows), at most 16. MDELAST_TPA
// overrides it.
int default_tpa(int n_atoms) {
    if (char const *e = std::getenv("MDELAST_TPA")) {
        int const v = std::atoi(e);
        if (valid_tpa(v))
            return v;
    }
    for (int t : {1, 4, 8})
        if (static_cast<long>(n_atoms) * t >= 150000)
            return t;
    return 16;
}

// Deal the blocks of a pair pass out to the replicas in proportion to their atom counts:
// about `target` in all (a multiple of the 148 SMs: a block then loops over several atom
// groups only for large batches), never fewer than one per replica nor more than one per
// atom group of kBlock/tpa atoms. Fills each replica's block range and the block ->
// replica map; returns the grid size.
constexpr int kTargetBlocks = 148 * 32;
// shared memory for the staged force tables: beside it the kernel keeps its FP64
// accumulators (40 KB at 4 lanes per atom) within the 227 KB a block may take
constexpr long kStageBudget = 184 * 1024;
// k_sublist grid: one wave, 5 resident blocks of 256 threads (48 registers each: 5 blocks
// fill the register file) on each of the 148 SMs
constexpr int kSublistBlocks = 148 * 5;

int deal_blocks(std::vector<Replica *> const &reps, int tpa, bool density,
                std::vector<int> &blk_rep, int target = kTargetBlocks,
                int block_threads = kBlock) {
    long total = 0;
    for (Replica const *r : reps)
        total += r->n_blocks;
    blk_rep.clear();
    for (size_t k = 0; k < reps.size(); ++k) {
        Replica *r = reps[k];
        // atom groups of block_threads / tpa atoms in the replica's kBlock-multiple range
        long const most = (static_cast<long>(r->n_blocks) * kBlock * tpa + block_threads - 1) /
                          block_threads;
        long nb = (static_cast<long>(target) * r->n_blocks + total - 1) / total;
        nb = std::max(1L, std::min(nb, most));
        if (density) {
            r->dblk_begin = static_cast<int>(blk_rep.size());
            r->dblk_n = static_cast<int>(nb);
        } else {
            r->fblk_begin = static_cast<int>(blk_rep.size());
            r->fblk_n = static_cast<int>(nb);
        }
        blk_rep.insert(blk_rep.end(), static_cast<size_t>(nb), static_cast<int>(k));
    }
    return static_cast<int>(blk_rep.size());
}

char const *fatal_message(unsigned bits) {
    if (bits & MDELAST_FATAL_RHO_MAX)
        return "FATAL: EAM F rho >rhomax_fatal";
    if (bits & MDELAST_FATAL_VOLUME)
        return "FATAL: volume change too large...";
    if (bits & MDELAST_FATAL_MOMENTUM)
        return "FATAL: total momentum";
    if (bits & MDELAST_FATAL_PRESSURE)
        return "FATAL PRESS";
    if (bits & MDELAST_FATAL_CONSERVATION)
        return "FATAL: bad energy conservation...";
    if (bits & MDELAST_ERR_LIST_OVERFLOW)
        return "neighbour list capacity exceeded";
    if (bits & MDELAST_ERR_CELL_OVERFLOW)
        return "cell list capacity exceeded";
    return "FATAL";
}

} // namespace

struct mdelast_driver_s {
    int device = 0;
    int smem_optin = 48 * 1024; // largest dynamic shared memory a block may opt into
    // k_nbr_cells for cell-list replicas (MDELAST_CELL_STAGING=0: k_nbr_build's per-atom
    // cell walk for all, which gives the same list)
    bool cell_staging = true;
    cudaStream_t stream = nullptr;
    int N = 0, n_pad = 0, n_rep = 1, ntypes = 0, npot = 0, n_blocks = 0;
    int tpa_d = 1, tpa_f = 1; // lanes per atom of the density and force passes
    int grid_d = 1, grid_f = 1; // blocks of the density and force passes
    int *d_dblk_rep = nullptr, *d_fblk_rep = nullptr;
    int neighbors = 0;
    double r_skin = 1., r_list = 0.;
    int sample = 1;
    bool stepped = false, obs_valid = false, dead = false;
    unsigned dead_bits = 0;

    Replica *d_rep = nullptr;
    int *d_rep_of = nullptr;
    double4 *d_crd = nullptr;
    double *d_vel = nullptr, *d_frc = nullptr, *d_rho = nullptr, *d_Fe = nullptr,
           *d_epot = nullptr;
    double2 *d_dF2 = nullptr;
    int precision = MDELAST_PRECISION_FP64;
    float4 *d_posf = nullptr;
    float2 *d_dF2f = nullptr;
    float *d_rbf = nullptr, *d_rrf = nullptr;
    void pass_density(bool obs, cudaStream_t s) {
        if (precision == MDELAST_PRECISION_MIXED)
            launch_density_mx(obs, tpa_d, grid_d, s, A, T);
        else
            launch_density(obs, tpa_d, grid_d, s, A, T);
    }
    // force pass with the staged shared-memory tables (mixed precision, quintic, when the
    // tables were staged; chosen by the autotuner or set_force_staging)
    bool stage_f = false;
    float *d_stf = nullptr;
    bool staging_available() const {
        return precision == MDELAST_PRECISION_MIXED && T.st_n > 0;
    }
    void pass_force(bool obs, bool kick, cudaStream_t s) {
        if (precision == MDELAST_PRECISION_MIXED && stage_f && T.st_n > 0)
            launch_force_mx_staged(obs, kick, tpa_f, grid_f, s, A, T);
        else if (precision == MDELAST_PRECISION_MIXED)
            launch_force_mx(obs, kick, tpa_f, grid_f, s, A, T);
        else
            launch_force(obs, kick, tpa_f, grid_f, s, A, T);
    }
    int *d_nbr = nullptr, *d_nup = nullptr, *d_ndn = nullptr;
    // pair list of the pair passes (see AtomsView::pnbr); pair_factor 0: the neighbour list
    int *d_pnbr = nullptr, *d_pnup = nullptr, *d_pndn = nullptr;
    // 16-bit entries (offsets within the replica) when every replica has at most 65,536
    // atoms; MDELAST_PAIR_LIST_16=0 keeps 32-bit entries
    uint16_t *d_pnbr16 = nullptr;
    bool pair16 = false;
    int alloc_pair_rows();
    double4 *d_crd_ref = nullptr;
    double pair_factor = 0., rcut0 = 0.;
    int set_pair_list(double factor);
    void point_pair_list();
    void refresh_pair_list(cudaStream_t s) {
        if (A.crd_ref) {
            size_t const smem = sublist_smem(A.maxn);
            if (smem > 48 * 1024)
                cudaFuncSetAttribute(k_sublist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem));
            k_sublist<<<std::min(n_pad / 8, kSublistBlocks), 256, smem, s>>>(A);
        }
    }
    double *d_pd = nullptr, *d_pf = nullptr, *d_red = nullptr;
    size_t cap_dmap = 0, cap_fmap = 0, cap_pd = 0, cap_pf = 0, cap_red = 0; // elements
    // closing scalar work: fold the block sums, then the per-replica kernel
    void post(int mode, int obs, cudaStream_t s) {
        k_reduce<<<dim3(A.max_chunks, n_rep), 256, 0, s>>>(A);
        k_post<<<n_rep, 256, 0, s>>>(A, mode, obs);
    }
    int *d_cell_count = nullptr, *d_cell_atoms = nullptr, *d_max_count = nullptr;
    int *d_halt = nullptr; // AtomsView::halt
    // The last launch of steps, for resuming it after a list build ran out of capacity in
    // one of its steps: cycle before it, steps, rebuild and sampling cadence.
    struct Launch {
        bool resumable = false;
        unsigned long long start = 0;
        int n = 0, rebuild_every = 0, sample_every = 0;
    } last_launch;
    int resume_after_overflow();
    int *d_cell_rep = nullptr;
    std::vector<int> cell_rep_host; // replica of each cell, as uploaded
    double *d_rb = nullptr, *d_Ft = nullptr;
    double *d_pos0 = nullptr, *d_out = nullptr;
    int *d_tmp_i = nullptr;
    size_t tmp_i_cap = 0;

    // sample rings: [n_rep][ring_cap] records; records of replica r already drained
    mdelast_sample *d_ring = nullptr;
    std::vector<long long> drained;
    int alloc_ring(int cap);
    // g(r) of each replica (md_driver.cpp:732-862): bin centres, results and counters on
    // the device; replica r's rg and gr start at gr_off[r], its partial rows at npot * gr_off[r]
    std::vector<long> gr_off;
    std::vector<int> gr_n;
    std::vector<double> gr_drg, gr_rmax;
    double *d_rg = nullptr, *d_gr = nullptr, *d_grp = nullptr;
    unsigned long long *d_gr_counts = nullptr;
    int *d_gr_ntype = nullptr;

    AtomsView A{};
    TablesView T{};
    mdelast_observables *h_obs = nullptr; // pinned, n_rep entries
    cudaEvent_t ev_step = nullptr;
    cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr}; // [2 * rebuild + obs]
    unsigned long long host_cycle = 0; // steps launched (the reference's cycle counter)
    int list_regrowths = 0;            // launches resumed after a list overflow
    bool all_pairs = false; // every replica lists by all-pairs search

    ~mdelast_driver_s();
    int alloc_list(int maxn);
    int alloc_cells(int n_cells, int cell_cap);
    void drop_graphs();
    int cells_alloc = 0;
    int configure_cells(std::vector<double> const &boxes); // 3 edges per replica
    std::vector<double> current_boxes() const;
    std::vector<int> rep_begin, rep_count; // atom slot range of each replica
    std::vector<long> pos0_off;            // offset of each replica in d_pos0
    int enqueue_rebuild();
    int build_list_checked();
    int enqueue_step(int obs, int rebuild, cudaEvent_t const *ev = nullptr);
    int time_steps(int n, int rebuild_every, double *ms_d, double *ms_f);
    int tune_on_steps(int n, int rebuild_every, int *choice, double *ms);
    int step_graph(int obs, int rebuild, cudaGraphExec_t *out);
    int launch_steps(int n_steps, int rebuild_every, int sample_every);
    int wait_step();
    int check_status();
    // launch shape of the pair passes: lanes per atom and target block counts
    int target_d = kTargetBlocks, target_f = kTargetBlocks;
    int set_launch(int tpa_d_, int tpa_f_, int tgt_d, int tgt_f, int staged = -1);
    int time_passes(int n_repeat, int obs, double *ms_d, double *ms_f);
};

mdelast_driver_s::~mdelast_driver_s() {
    if (device >= 0)
        cudaSetDevice(device);
    for (auto &g : graph)
        if (g)
            cudaGraphExecDestroy(g);
    if (ev_step)
        cudaEventDestroy(ev_step);
    if (h_obs)
        cudaFreeHost(h_obs);
    dfree(d_rep);
    dfree(d_rep_of);
    dfree(d_crd);
    dfree(d_vel);
    dfree(d_frc);
    dfree(d_rho);
    dfree(d_Fe);
    dfree(d_epot);
    dfree(d_dF2);
    dfree(d_posf);
    dfree(d_dF2f);
    dfree(d_rbf);
    dfree(d_rrf);
    dfree(d_stf);
    dfree(d_nbr);
    dfree(d_nup);
    dfree(d_ndn);
    dfree(d_pnbr);
    dfree(d_pnbr16);
    dfree(d_pnup);
    dfree(d_pndn);
    dfree(d_crd_ref);
    dfree(d_pd);
    dfree(d_pf);
    dfree(d_red);
    dfree(d_cell_count);
    dfree(d_cell_atoms);
    dfree(d_cell_rep);
    dfree(d_max_count);
    dfree(d_halt);
    dfree(d_rb);
    dfree(d_Ft);
    dfree(d_pos0);
    dfree(d_out);
    dfree(d_tmp_i);
    dfree(d_dblk_rep);
    dfree(d_fblk_rep);
    dfree(d_ring);
    dfree(d_rg);
    dfree(d_gr);
    dfree(d_grp);
    dfree(d_gr_counts);
    dfree(d_gr_ntype);
    if (stream)
        cudaStreamDestroy(stream);
}

int mdelast_driver_s::alloc_list(int maxn) {
    dfree(d_nbr);
    if (int rc = dalloc(&d_nbr, static_cast<size_t>(maxn) * n_pad))
        return rc;
    A.nbr = d_nbr;
    A.maxn = maxn;
    if (pair_factor > 0.)
        if (int rc = alloc_pair_rows())
            return rc;
    point_pair_list();
    drop_graphs();
    return MDELAST_OK;
}

// rows of the pair list at the neighbour list's capacity, in the chosen entry width
int mdelast_driver_s::alloc_pair_rows() {
    dfree(d_pnbr);
    dfree(d_pnbr16);
    size_t const n = static_cast<size_t>(A.maxn) * n_pad;
    return pair16 ? dalloc(&d_pnbr16, n) : dalloc(&d_pnbr, n);
}

void mdelast_driver_s::point_pair_list() {
    A.pnbr16 = nullptr;
    if (pair_factor > 0.) {
        A.pnbr = d_pnbr;
        A.pnbr16 = pair16 ? d_pnbr16 : nullptr;
        A.pn_up = d_pnup;
        A.pn_dn = d_pndn;
        A.crd_ref = d_crd_ref;
        double const rs = pair_factor * rcut0, half = 0.5 * (pair_factor - 1.) * rcut0;
        A.sub_r2 = rs * rs;
        A.sub_half2 = half * half;
    } else {
        A.pnbr = A.nbr;
        A.pn_up = A.n_up;
        A.pn_dn = A.n_dn;
        A.crd_ref = nullptr;
        A.sub_r2 = A.sub_half2 = 0.;
    }
    A.pmaxn = A.maxn;
}

// The pair passes read the neighbour list's pairs within factor * r_cut, refreshed when
// needed (factor 0: the neighbour list itself). Rebuilds the rows now.
int mdelast_driver_s::set_pair_list(double factor) {
    if (factor != 0. && !(factor > 1.))
        return fail(MDELAST_ERR_ARGUMENT, "pair-list radius factor must be 0 or > 1");
    if (!neighbors || factor >= r_skin)
        factor = 0.; // without a neighbour list, or no tighter than it: nothing to gain
    CK(cudaStreamSynchronize(stream));
    drop_graphs();
    dfree(d_pnbr);
    dfree(d_pnbr16);
    dfree(d_pnup);
    dfree(d_pndn);
    dfree(d_crd_ref);
    pair_factor = factor;
    {
        int most = 0;
        for (int c : rep_count)
            most = std::max(most, c);
        char const *e = std::getenv("MDELAST_PAIR_LIST_16");
        pair16 = most <= 65536 && !(e && std::atoi(e) == 0);
    }
    if (factor > 0.) {
        if (int rc = alloc_pair_rows())
            return rc;
        if (int rc = dalloc(&d_pnup, static_cast<size_t>(n_pad)))
            return rc;
        if (int rc = dalloc(&d_pndn, static_cast<size_t>(n_pad)))
            return rc;
        if (int rc = dalloc(&d_crd_ref, static_cast<size_t>(n_pad)))
            return rc;
    }
    point_pair_list();
    if (A.crd_ref) {
        k_sub_invalidate<<<1, 128, 0, stream>>>(A);
        refresh_pair_list(stream);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(stream));
    }
    return MDELAST_OK;
}

int mdelast_driver_s::alloc_cells(int n_cells, int cell_cap) {
    dfree(d_cell_count);
    dfree(d_cell_atoms);
    dfree(d_cell_rep);
    cell_rep_host.clear();
    if (int rc = dalloc(&d_cell_count, static_cast<size_t>(std::max(n_cells, 1))))
        return rc;
    if (int rc = dalloc(&d_cell_rep, static_cast<size_t>(std::max(n_cells, 1))))
        return rc;
    A.cell_rep = d_cell_rep;
    if (int rc = dalloc(&d_cell_atoms, static_cast<size_t>(std::max(n_cells, 1)) * cell_cap))
        return rc;
    A.cell_count = d_cell_count;
    A.cell_atoms = d_cell_atoms;
    cells_alloc = n_cells;
    A.cell_cap = cell_cap;
    drop_graphs();
    return MDELAST_OK;
}

// Re-deal the pair-pass blocks for new lanes-per-atom and block targets: replica block
// ranges, block -> replica maps, per-block and per-chunk partial-sum buffers. The step
// graphs hold the old shapes and are dropped. Call with no work in flight.
int mdelast_driver_s::set_launch(int tpa_d_, int tpa_f_, int tgt_d, int tgt_f, int staged) {
    if (!valid_tpa(tpa_d_) || !valid_tpa(tpa_f_) || tgt_d < 1 || tgt_f < 1)
        return fail(MDELAST_ERR_ARGUMENT, "bad launch shape");
    bool const st = staged < 0 ? stage_f : staged != 0;
    if (st && !staging_available())
        return fail(MDELAST_ERR_UNSUPPORTED,
                    "staged force tables need mixed precision and quintic tables that fit");
    if (st && tpa_f_ == 1)
        return fail(MDELAST_ERR_ARGUMENT, "the staged force pass takes 4, 8 or 16 lanes per atom");
    CK(cudaStreamSynchronize(stream));
    std::vector<Replica> R(static_cast<size_t>(n_rep));
    CK(cudaMemcpy(R.data(), d_rep, sizeof(Replica) * n_rep, cudaMemcpyDeviceToHost));
    std::vector<Replica *> reps;
    for (auto &x : R)
        reps.push_back(&x);
    std::vector<int> dmap, fmap;
    int const gd = deal_blocks(reps, tpa_d_, true, dmap, tgt_d);
    int const gf = deal_blocks(reps, tpa_f_, false, fmap, tgt_f, st ? kStagedBlock : kBlock);
    int chunks = 1;
    for (Replica const *x : reps)
        chunks = std::max(chunks, (std::max(x->dblk_n, x->fblk_n) + kChunk - 1) / kChunk);
    drop_graphs();
    // grow the block maps and sums only: the autotuner tries many shapes in a row, and a
    // free and an allocation per shape cost far more than the launches it times
    auto grow = [](auto *&p, size_t &cap, size_t n) -> int {
        if (n <= cap && p)
            return MDELAST_OK;
        dfree(p);
        cap = 0;
        if (int rc = dalloc(&p, n))
            return rc;
        cap = n;
        return MDELAST_OK;
    };
    if (int rc = grow(d_dblk_rep, cap_dmap, dmap.size()))
        return rc;
    if (int rc = grow(d_fblk_rep, cap_fmap, fmap.size()))
        return rc;
    if (int rc = grow(d_pd, cap_pd, static_cast<size_t>(gd) * D_NSUM))
        return rc;
    if (int rc = grow(d_pf, cap_pf, static_cast<size_t>(gf) * F_NSUM))
        return rc;
    if (int rc = grow(d_red, cap_red, static_cast<size_t>(n_rep) * chunks * 64))
        return rc;
    CK(cudaMemcpy(d_dblk_rep, dmap.data(), sizeof(int) * dmap.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_fblk_rep, fmap.data(), sizeof(int) * fmap.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_rep, R.data(), sizeof(Replica) * n_rep, cudaMemcpyHostToDevice));
    tpa_d = tpa_d_;
    tpa_f = tpa_f_;
    target_d = tgt_d;
    target_f = tgt_f;
    stage_f = st;
    grid_d = gd;
    grid_f = gf;
    A.dblk_rep = d_dblk_rep;
    A.fblk_rep = d_fblk_rep;
    A.pd = d_pd;
    A.pf = d_pf;
    A.red = d_red;
    A.max_chunks = chunks;
    return MDELAST_OK;
}

// n real steps, launched one by one with events around the two pair passes (the state
// advances exactly as in run(n, rebuild_every, 1)); mean device time of the density and
// the force pass over them. The passes then run in the cache state a step leaves them,
// which repeated passes on a fixed state do not reproduce.
int mdelast_driver_s::time_steps(int n, int rebuild_every, double *ms_d, double *ms_f) {
    cudaEvent_t ev[3];
    for (auto &e : ev)
        CK(cudaEventCreate(&e));
    double td = 0., tf = 0.;
    int rc = MDELAST_OK;
    for (int k = 0; k < n && !rc; ++k) {
        unsigned long long const c = host_cycle;
        int const rebuild = neighbors && rebuild_every > 0 &&
                            c % static_cast<unsigned>(rebuild_every) == 0;
        // a one-step launch, resumable like run()'s after a list overflow
        last_launch.resumable = neighbors && rebuild_every > 0;
        last_launch.start = c;
        last_launch.n = 1;
        last_launch.rebuild_every = rebuild_every;
        last_launch.sample_every = 1;
        rc = enqueue_step(1, rebuild, ev);
        if (rc)
            break;
        ++host_cycle;
        cudaError_t const e = cudaEventRecord(ev_step, stream);
        if (e != cudaSuccess) {
            rc = fail(MDELAST_ERR_CUDA, "step timing: %s", cudaGetErrorString(e));
            break;
        }
        obs_valid = false;
        stepped = true;
        rc = wait_step();
        if (rc)
            break;
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, ev[0], ev[1]);
        cudaEventElapsedTime(&b, ev[1], ev[2]);
        td += a;
        tf += b;
    }
    for (auto &e : ev)
        cudaEventDestroy(e);
    if (rc)
        return rc;
    *ms_d = td / n;
    *ms_f = tf / n;
    return MDELAST_OK;
}

// The launch shapes timed on real steps (time_steps): first the density pass over its
// shapes with the force shape fixed, then the force pass (both variants) with the best
// density shape; n steps per shape.
int mdelast_driver_s::tune_on_steps(int n, int rebuild_every, int *choice, double *ms) {
    double best_d = 1e300, best_f = 1e300;
    int bd[2] = {tpa_d, target_d}, bf[3] = {tpa_f, target_f, stage_f ? 1 : 0};
    for (int tp : {1, 4, 8, 16})
        for (int tg : {148 * 16, 148 * 32, 148 * 64}) {
            if (int rc = set_launch(tp, bf[0], tg, bf[1], bf[2]))
                return rc;
            double md = 0., mf = 0.;
            if (int rc = time_steps(n, rebuild_every, &md, &mf))
                return rc;
            if (md < best_d) {
                best_d = md;
                bd[0] = tp;
                bd[1] = tg;
            }
        }
    struct Shape {
        int tpa, target, staged;
    };
    std::vector<Shape> shapes;
    for (int tp : {1, 4, 8, 16})
        for (int tg : {148 * 8, 148 * 16, 148 * 32})
            shapes.push_back({tp, tg, 0});
    if (staging_available())
        for (int tp : {4, 8})
            for (int tg : {148 * 4, 148 * 8})
                shapes.push_back({tp, tg, 1});
    for (Shape const &x : shapes) {
        if (int rc = set_launch(bd[0], x.tpa, bd[1], x.target, x.staged))
            return rc;
        double md = 0., mf = 0.;
        if (int rc = time_steps(n, rebuild_every, &md, &mf))
            return rc;
        if (mf < best_f) {
            best_f = mf;
            bf[0] = x.tpa;
            bf[1] = x.target;
            bf[2] = x.staged;
        }
    }
    if (int rc = set_launch(bd[0], bf[0], bd[1], bf[1], bf[2]))
        return rc;
    choice[0] = bd[0];
    choice[1] = bf[0];
    choice[2] = bd[1];
    choice[3] = bf[1];
    ms[0] = best_d;
    ms[1] = best_f;
    return MDELAST_OK;
}

// Mean device time of the density and the force pass (no kick: the state is unchanged)
// over n_repeat launches on the current positions, after one untimed pair.
int mdelast_driver_s::time_passes(int n_repeat, int obs, double *ms_d, double *ms_f) {
    cudaEvent_t ev[3];
    for (auto &e : ev)
        CK(cudaEventCreate(&e));
    double td = 0., tf = 0.;
    cudaError_t err = cudaSuccess;
    for (int k = 0; k <= n_repeat && err == cudaSuccess; ++k) {
        cudaEventRecord(ev[0], stream);
        pass_density(obs != 0, stream);
        cudaEventRecord(ev[1], stream);
        pass_force(obs != 0, false, stream);
        cudaEventRecord(ev[2], stream);
        err = cudaEventSynchronize(ev[2]);
        if (err == cudaSuccess && k > 0) {
            float a = 0.f, b = 0.f;
            cudaEventElapsedTime(&a, ev[0], ev[1]);
            cudaEventElapsedTime(&b, ev[1], ev[2]);
            td += a;
            tf += b;
        }
    }
    for (auto &e : ev)
        cudaEventDestroy(e);
    if (err != cudaSuccess)
        return fail(MDELAST_ERR_CUDA, "pass timing: %s", cudaGetErrorString(err));
    *ms_d = td / n_repeat;
    *ms_f = tf / n_repeat;
    return MDELAST_OK;
}

int mdelast_driver_s::alloc_ring(int cap) {
    drop_graphs(); // the step graphs hold the ring pointer
    dfree(d_ring);
    A.ring = nullptr;
    A.ring_cap = 0;
    if (cap > 0) {
        if (int rc = dalloc(&d_ring, static_cast<size_t>(n_rep) * cap))
            return rc;
        A.ring = d_ring;
        A.ring_cap = cap;
    }
    drained.assign(static_cast<size_t>(n_rep), 0);
    k_samples_reset<<<(n_rep + 63) / 64, 64, 0, stream>>>(A, 1);
    CK(cudaGetLastError());
    // complete before any host-side read-modify-write of the replica states
    CK(cudaStreamSynchronize(stream));
    return MDELAST_OK;
}

void mdelast_driver_s::drop_graphs() {
    for (auto &g : graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// Half cells per edge for the current box: twice the number of cells no thinner than the
// list radius (with a margin for the box changes of an NPT run between rebuilds); fewer
// than 3 such cells along any edge means an all-pairs search.
int mdelast_driver_s::configure_cells(std::vector<double> const &boxes) {
    // per replica: cells per edge from its box, and its block of the global cell arrays
    std::vector<Replica> R(static_cast<size_t>(n_rep));
    CK(cudaMemcpy(R.data(), d_rep, sizeof(Replica) * n_rep, cudaMemcpyDeviceToHost));
    bool changed = false, all_brute = true;
    int n_cells = 0, cap = std::max(A.cell_cap, 32);
    for (int q = 0; q < n_rep; ++q) {
        int nc[3];
        bool brute = false;
        for (int a = 0; a < 3; ++a) {
            nc[a] = static_cast<int>(std::floor(boxes[3 * q + a] / (r_list * 1.05)));
            if (nc[a] < 3)
                brute = true;
            nc[a] *= 2;
        }
        if (brute)
            nc[0] = nc[1] = nc[2] = 0;
        Replica &r = R[static_cast<size_t>(q)];
        if (r.nc[0] != nc[0] || r.nc[1] != nc[1] || r.nc[2] != nc[2] || r.cell_begin != n_cells)
            changed = true;
        r.nc[0] = nc[0];
        r.nc[1] = nc[1];
        r.nc[2] = nc[2];
        r.cell_begin = n_cells;
        int const nq = brute ? 0 : nc[0] * nc[1] * nc[2];
        if (nq > 0)
            cap = std::max(cap, static_cast<int>(2. * r.n_atoms / nq) + 16);
        n_cells += nq;
        all_brute = all_brute && brute;
    }
    if (changed)
        CK(cudaMemcpy(d_rep, R.data(), sizeof(Replica) * n_rep, cudaMemcpyHostToDevice));
    if (!d_cell_count || n_cells > cells_alloc || cap > A.cell_cap)
        if (int rc = alloc_cells(std::max(n_cells, cells_alloc), cap))
            return rc;
    std::vector<int> crep;
    for (int q = 0; q < n_rep; ++q) {
        Replica const &x = R[static_cast<size_t>(q)];
        if (x.nc[0] > 0)
            crep.insert(crep.end(), static_cast<size_t>(x.nc[0]) * x.nc[1] * x.nc[2], q);
    }
    if (crep != cell_rep_host) {
        if (!crep.empty())
            CK(cudaMemcpy(d_cell_rep, crep.data(), sizeof(int) * crep.size(),
                          cudaMemcpyHostToDevice));
        cell_rep_host = crep;
    }
    if (changed || all_pairs != all_brute || A.n_cells != n_cells)
        drop_graphs(); // the launch shape of the cell kernels is part of the graphs
    all_pairs = all_brute;
    A.n_cells = n_cells;
    return MDELAST_OK;
}

std::vector<double> mdelast_driver_s::current_boxes() const {
    std::vector<double> b;
    for (int q = 0; q < n_rep; ++q)
        for (int a = 0; a < 3; ++a)
            b.push_back(h_obs[q].box[4 * a]);
    return b;
}

int mdelast_driver_s::enqueue_rebuild() {
    CK(cudaMemsetAsync(d_max_count, 0, 2 * sizeof(int), stream));
    int const grid = n_pad / kBlock;
    if (!all_pairs && A.n_cells > 0) {
        CK(cudaMemsetAsync(d_cell_count, 0, sizeof(int) * A.n_cells, stream));
        k_cell_bin<<<grid, kBlock, 0, stream>>>(A);
        // one warp per half cell, as many per block as their scratch (cell_cap ints each)
        // fits; a capacity beyond one warp's share fails here rather than at the launch
        size_t const per_warp = sizeof(int) * static_cast<size_t>(A.cell_cap);
        int const wpb = static_cast<int>(
            std::min<size_t>(kCellSortWarps, static_cast<size_t>(smem_optin - 64) / per_warp));
        if (wpb < 1)
            return fail(MDELAST_ERR_CAPACITY, "cell capacity %d exceeds the shared memory of "
                        "the cell sort", A.cell_cap);
        size_t const sort_smem = per_warp * wpb;
        if (sort_smem > 48 * 1024)
            CK(cudaFuncSetAttribute(k_cell_sort, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(sort_smem)));
        k_cell_sort<<<(A.n_cells + wpb - 1) / wpb, 32 * wpb, sort_smem, stream>>>(A);
    }
    int cells_done = 0;
    size_t const smem = nbr_cells_smem(A.cell_cap);
    // cells so crowded that a group's staging does not fit: k_nbr_build walks the cells
    if (cell_staging && !all_pairs && A.n_cells > 0 &&
        smem + kNbrCellsStaticSmem <= static_cast<size_t>(smem_optin)) {
        // the dynamic part alone may stay below 48 KB while static + dynamic exceed it
        CK(cudaFuncSetAttribute(k_nbr_cells, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(smem)));
        k_nbr_cells<<<A.n_cells / 8, kNbrCellsThreads, smem, stream>>>(A);
        cells_done = 1;
    }
    // all-pairs replicas, and cell replicas k_nbr_cells left (narrow or too crowded cells)
    k_nbr_build<<<std::min(n_pad / 8, 148 * 8), 256, 0, stream>>>(A, cells_done);
    if (A.crd_ref)
        k_sub_invalidate<<<1, 128, 0, stream>>>(A);
    CK(cudaGetLastError());
    return MDELAST_OK;
}

// Headroom of neighbour-list capacities: a new capacity is (1 + h) times the largest count
// plus 32 (plus nothing when h is 0); MDELAST_LIST_HEADROOM sets h (default 0.5).
double list_headroom() {
    if (char const *e = std::getenv("MDELAST_LIST_HEADROOM")) {
        double const h = std::atof(e);
        if (h >= 0. && h <= 16.)
            return h;
    }
    return 0.5;
}

// Build the list now and grow the neighbour or cell capacity until it fits.
int mdelast_driver_s::build_list_checked() {
    for (int attempt = 0; attempt < 6; ++attempt) {
        if (int rc = enqueue_rebuild())
            return rc;
        int mc[2];
        CK(cudaMemcpyAsync(mc, d_max_count, sizeof(mc), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        bool grow = false;
        if (mc[1] > A.cell_cap) {
            if (int rc = alloc_cells(cells_alloc, mc[1] + mc[1] / 2 + 32))
                return rc;
            grow = true;
        }
        if (mc[0] > A.maxn) {
            double const h = list_headroom();
            int const m = (static_cast<int>(mc[0] * (1. + h)) + (h > 0. ? 32 : 0) + 3) / 4 * 4;
            if (int rc = alloc_list(std::max(m, mc[0])))
                return rc;
            grow = true;
        }
        if (!grow) {
            CK(cudaMemsetAsync(d_halt, 0, sizeof(int), stream));
            return MDELAST_OK;
        }
        // the overflow bits of the attempt that did not fit
        k_status_and<<<1, 32, 0, stream>>>(A, ~(MDELAST_ERR_LIST_OVERFLOW | MDELAST_ERR_CELL_OVERFLOW));
        CK(cudaGetLastError());
    }
    return fail(MDELAST_ERR_CAPACITY, "neighbour list did not fit after repeated growth");
}

int mdelast_driver_s::enqueue_step(int obs, int rebuild, cudaEvent_t const *ev) {
    int const grid = n_pad / kBlock;
    if (rebuild && neighbors) // calculate_neighbors() before integrate() (md.py:1245-1251)
        if (int rc = enqueue_rebuild())
            return rc;
    k_pre<<<n_rep, 64, 0, stream>>>(A);
    k_kick_drift<<<grid, kBlock, 0, stream>>>(A, T);
    if (!neighbors)
        if (int rc = enqueue_rebuild())
            return rc;
    refresh_pair_list(stream);
    if (ev)
        CK(cudaEventRecord(ev[0], stream));
    pass_density(obs != 0, stream);
    if (ev)
        CK(cudaEventRecord(ev[1], stream));
    pass_force(obs != 0, true, stream);
    if (ev)
        CK(cudaEventRecord(ev[2], stream));
    post(POST_STEP, obs, stream);
    CK(cudaGetLastError());
    CK(cudaMemcpy2DAsync(h_obs, sizeof(mdelast_observables),
                         reinterpret_cast<char *>(d_rep) + offsetof(Replica, obs), sizeof(Replica),
                         sizeof(mdelast_observables), n_rep, cudaMemcpyDeviceToHost, stream));
    return MDELAST_OK;
}

// The instantiated graph of one step, captured on first use.
int mdelast_driver_s::step_graph(int obs, int rebuild, cudaGraphExec_t *out) {
    cudaGraphExec_t &ge = graph[2 * (rebuild ? 1 : 0) + (obs ? 1 : 0)];
    if (!ge) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_step(obs, rebuild);
        cudaError_t e = cudaStreamEndCapture(stream, &g);
        if (rc)
            return rc;
        if (e != cudaSuccess)
            return fail(MDELAST_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess)
            return fail(MDELAST_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    *out = ge;
    return MDELAST_OK;
}

// Launch n steps; rebuild_every / sample_every < 0 mean "never" / "use the flag".
int mdelast_driver_s::launch_steps(int n_steps, int rebuild_every, int sample_every) {
    last_launch.resumable = neighbors && rebuild_every > 0;
    last_launch.start = host_cycle;
    last_launch.n = n_steps;
    last_launch.rebuild_every = rebuild_every;
    last_launch.sample_every = sample_every;
    for (int s = 0; s < n_steps; ++s) {
        unsigned long long const c = host_cycle;
        int const rebuild = rebuild_every > 0 && c % static_cast<unsigned>(rebuild_every) == 0;
        int const obs = sample_every < 0 ? sample
                                         : (sample_every > 0 &&
                                            (c + 1) % static_cast<unsigned>(sample_every) == 0);
        cudaGraphExec_t g;
        if (int rc = step_graph(obs, rebuild, &g))
            return rc;
        CK(cudaGraphLaunch(g, stream));
        ++host_cycle;
    }
    if (n_steps > 0) {
        CK(cudaEventRecord(ev_step, stream));
        obs_valid = false;
        stepped = true;
    }
    return MDELAST_OK;
}

int mdelast_driver_s::wait_step() {
    if (!obs_valid) {
        CK(cudaEventSynchronize(ev_step));
        obs_valid = true;
    }
    return check_status();
}

// An in-step list rebuild ran out of neighbour or cell capacity (as the reference's list
// grows, md_driver.cpp:288-292): the kernels of that step and of every later step of the
// launch returned without work. Grow the capacity, rebuild at the unchanged positions and
// launch the remaining steps again, until the launch completes.
int mdelast_driver_s::resume_after_overflow() {
    unsigned const bits = MDELAST_ERR_LIST_OVERFLOW | MDELAST_ERR_CELL_OVERFLOW;
    for (int attempt = 0; attempt < 64; ++attempt) {
        bool over = false;
        for (int r = 0; r < n_rep; ++r)
            over = over || (h_obs[r].status & bits) != 0;
        if (!over)
            return MDELAST_OK;
        if (!last_launch.resumable)
            return MDELAST_OK; // reported as fatal by check_status
        // every replica completed the same steps: their cycle counters agree
        unsigned long long const done = static_cast<unsigned long long>(h_obs[0].cycle);
        if (done < last_launch.start || done > last_launch.start + last_launch.n)
            return fail(MDELAST_ERR_CUDA, "inconsistent cycle after a list overflow");
        int const left = static_cast<int>(last_launch.start + last_launch.n - done);
        k_status_and<<<1, 32, 0, stream>>>(A, ~bits);
        CK(cudaGetLastError());
        for (int r = 0; r < n_rep; ++r)
            h_obs[r].status &= ~bits;
        host_cycle = done;
        if (int rc = configure_cells(current_boxes()))
            return rc;
        if (int rc = build_list_checked()) // grows, rebuilds and clears the halt
            return rc;
        if (int rc = launch_steps(left, last_launch.rebuild_every, last_launch.sample_every))
            return rc;
        CK(cudaEventSynchronize(ev_step));
        ++list_regrowths;
    }
    return fail(MDELAST_ERR_CAPACITY, "neighbour list kept overflowing after repeated growth");
}

int mdelast_driver_s::check_status() {
    if (dead)
        return fail(MDELAST_ERR_FATAL, "%s (status 0x%x)", fatal_message(dead_bits), dead_bits);
    if (int rc = resume_after_overflow())
        return rc;
    for (int r = 0; r < n_rep; ++r) {
        unsigned const st = h_obs[r].status;
        if (st & MDELAST_FATAL_MASK) {
            dead = true;
            dead_bits = st;
            return fail(MDELAST_ERR_FATAL, "%s (status 0x%x)", fatal_message(st), st);
        }
    }
    return MDELAST_OK;
}

extern "C" {

int mdelast_release_cached_memory(int32_t device) {
    clear_error();
    int n = 0;
    CK(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n)
        return fail(MDELAST_ERR_ARGUMENT, "device %d out of range", device);
    CK(cudaSetDevice(device));
    CK(cudaDeviceSynchronize());
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pool_mutex);
        if (static_cast<size_t>(device) < g_pools.size())
            pool = g_pools[static_cast<size_t>(device)];
    }
    if (pool)
        CK(cudaMemPoolTrimTo(pool, 0));
    {
        std::lock_guard<std::mutex> lock(g_stage_mutex);
        if (g_stage)
            cudaFreeHost(g_stage);
        g_stage = nullptr;
        g_stage_bytes = 0;
    }
    return MDELAST_OK;
}

int mdelast_device_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n > 0;
}

} // extern "C"

// Validate one replica's configuration against the shared tables (those of replica 0).
static int check_config(mdelast_driver_config const &c, mdelast_driver_config const &c0, int r) {
    int const N = c.n_atoms, nt = c.n_types;
    if (N < 2 || nt < 1 || nt > kMaxTypes)
        return fail(MDELAST_ERR_ARGUMENT, "replica %d: need n_atoms >= 2 and 1 <= n_types <= %d",
                    r, kMaxTypes);
    if (!c.positions || !c.velocities || !c.types || !c.mass || !c.pair)
        return fail(MDELAST_ERR_ARGUMENT, "replica %d: null array in the configuration", r);
    int const npot = nt * (nt + 1) / 2;
    if (c.n_eam != 0 && c.n_eam != nt)
        return fail(MDELAST_ERR_ARGUMENT, "EAM objects: %d given, %d types", c.n_eam, nt);
    if (c.ensemble < MDELAST_NVE || c.ensemble > MDELAST_NPT)
        return fail(MDELAST_ERR_UNSUPPORTED, "bad ensamble %d", c.ensemble);
    if (c.coupling < 0 || c.coupling > 2)
        return fail(MDELAST_ERR_ARGUMENT, "bad thermostat coupling %d", c.coupling);
    if (!(c.dt > 0.) || !(c.r_skin >= 1.))
        return fail(MDELAST_ERR_ARGUMENT, "need dt > 0 and r_skin >= 1");
    if (c.thermo_nchain < 1 || c.thermo_nchain > kMaxChain || c.baro_nchain < 1 ||
        c.baro_nchain > kMaxChain || !c.thermo_q || !c.thermo_p_eta || !c.baro_q ||
        !c.baro_p_eta)
        return fail(MDELAST_ERR_ARGUMENT, "thermostat chains need 1..%d links", kMaxChain);
    if (c.n_rg < 2 || !c.rg)
        return fail(MDELAST_ERR_ARGUMENT, "rg needs at least 2 bins");
    if (!(c.rg[0] > 0.) || !(c.rg[1] > c.rg[0])) // md_driver.cpp:86-87
        return fail(MDELAST_ERR_ARGUMENT, "rg must be cell centred: rg[0] > 0, rg[1] > rg[0]");
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            if (a != b && c.box[3 * a + b] != 0.)
                return fail(MDELAST_ERR_ARGUMENT, "the box must be diagonal");
    if (c.precision != MDELAST_PRECISION_FP64 && c.precision != MDELAST_PRECISION_MIXED)
        return fail(MDELAST_ERR_ARGUMENT, "precision %d is not defined", c.precision);
    // tables: every pair slot and EAM function on one r grid
    mdelast_pair const *p0 = c.pair[0];
    for (int s = 0; s < npot; ++s) {
        mdelast_pair const *p = c.pair[s];
        if (!p)
            return fail(MDELAST_ERR_ARGUMENT, "pair slot %d is null", s);
        if (p->kind != PAIR_TABLE)
            return fail(MDELAST_ERR_UNSUPPORTED,
                        "analytic pair potentials (Morse, LennardJones) are not available on "
                        "the GPU path; tabulate them as TablePotential");
        if (p->table.n != p0->table.n || p->table.h != p0->table.h)
            return fail(MDELAST_ERR_UNSUPPORTED, "pair tables on different grids");
        if (p->interpolation != p0->interpolation)
            return fail(MDELAST_ERR_UNSUPPORTED,
                        "pair tables with different interpolations ('quintic', 'bspline')");
    }
    for (int t = 0; t < c.n_eam; ++t) {
        mdelast_eam const *e = c.eam[t];
        if (!e)
            return fail(MDELAST_ERR_ARGUMENT, "EAM %d is null", t);
        if (e->rho.n != p0->table.n || e->rho.h != p0->table.h ||
            e->F.n != c.eam[0]->F.n || e->F.h != c.eam[0]->F.h)
            return fail(MDELAST_ERR_UNSUPPORTED, "EAM tables on different grids");
        if (e->interpolation != p0->interpolation)
            return fail(MDELAST_ERR_UNSUPPORTED,
                        "EAM and pair tables with different interpolations");
    }
    if (r > 0) { // a batch shares the tables, the list settings, the precision and the device
        bool same = c.n_types == c0.n_types && c.n_eam == c0.n_eam &&
                    c.neighbors == c0.neighbors && c.r_skin == c0.r_skin &&
                    c.precision == c0.precision && c.device == c0.device;
        for (int s = 0; same && s < npot; ++s)
            same = c.pair[s] == c0.pair[s];
        for (int t = 0; same && t < c.n_eam; ++t)
            same = c.eam[t] == c0.eam[t];
        for (int t = 0; same && t < nt; ++t)
            same = c.mass[t] == c0.mass[t];
        if (!same)
            return fail(MDELAST_ERR_ARGUMENT,
                        "replica %d: a batch shares potentials, masses, list settings, "
                        "precision and device with replica 0", r);
    }
    return MDELAST_OK;
}

static void set_chain(Chain &ch, double T_, int n, const double *q, const double *p, double Nf) {
    ch.T = T_;
    ch.Nf = Nf;
    ch.n = n;
    for (int j = 0; j < n; ++j) {
        ch.q[j] = q[j];
        ch.inv_q[j] = 1. / q[j];
        ch.p_eta[j] = p[j];
        ch.eta[j] = 0.;
    }
}

// A system of n_rep independent replicas sharing one potential (n_rep = 1: MDDriver).
static int create_system(const mdelast_driver_config *cfgs, int n_rep, mdelast_driver **out) {
    clear_error();
    if (!cfgs || !out || n_rep < 1)
        return fail(MDELAST_ERR_ARGUMENT, "null argument or no replica");
    *out = nullptr;
    mdelast_driver_config const &c0 = cfgs[0];
    for (int r = 0; r < n_rep; ++r)
        if (int rc = check_config(cfgs[r], c0, r))
            return rc;
    int const nt = c0.n_types, npot = nt * (nt + 1) / 2;
    // scaled coordinates (md_driver.cpp:91-106) of every replica, packed at kTile offsets
    std::vector<int> begin(static_cast<size_t>(n_rep)), count(static_cast<size_t>(n_rep));
    int np = 0;
    long n_total = 0;
    for (int r = 0; r < n_rep; ++r) {
        begin[r] = np;
        count[r] = cfgs[r].n_atoms;
        np += (cfgs[r].n_atoms + kTile - 1) / kTile * kTile;
        n_total += cfgs[r].n_atoms;
    }
    for (int r = 0; r < n_rep; ++r) {
        mdelast_driver_config const &c = cfgs[r];
        double const L[3] = {c.box[0], c.box[4], c.box[8]};
        for (int a = 0; a < c.n_atoms; ++a) {
            double const *p = c.positions + 3 * a;
            if (std::abs(p[0]) >= 0.5 * L[0] || std::abs(p[1]) >= 0.5 * L[1] ||
                std::abs(p[2]) >= 0.5 * L[2])
                return fail(MDELAST_ERR_ARGUMENT, "bad initial position (replica %d atom %d)", r, a);
            if (c.types[a] >= static_cast<uint32_t>(nt))
                return fail(MDELAST_ERR_ARGUMENT, "bad type (replica %d atom %d)", r, a);
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(MDELAST_ERR_NO_DEVICE, "no CUDA device: the mdelast GPU path needs one");
    }
    if (c0.device < 0 || c0.device >= ndev)
        return fail(MDELAST_ERR_ARGUMENT, "device %d not present (%d devices)", c0.device, ndev);
    CK(cudaSetDevice(c0.device));
    // scaled coordinates and type, velocities (SoA), replica of each slot, and the initial
    // positions, written straight into the pinned staging that uploads them
    std::unique_lock<std::mutex> stage_lock(g_stage_mutex);
    size_t const b_crd = sizeof(double4) * static_cast<size_t>(np),
                 b_vel = sizeof(double) * 3 * static_cast<size_t>(np),
                 b_pos0 = sizeof(double) * 3 * static_cast<size_t>(n_total),
                 b_rep = sizeof(int) * static_cast<size_t>(np);
    char *stage = static_cast<char *>(stage_host(b_crd + b_vel + b_pos0 + b_rep));
    if (!stage)
        return fail(MDELAST_ERR_CUDA, "pinned host staging allocation failed");
    double4 *crd = reinterpret_cast<double4 *>(stage);
    double *vel = reinterpret_cast<double *>(stage + b_crd);
    double *pos0 = reinterpret_cast<double *>(stage + b_crd + b_vel);
    int *rep_of = reinterpret_cast<int *>(stage + b_crd + b_vel + b_pos0);
    long p0off = 0;
    for (int r = 0; r < n_rep; ++r) {
        mdelast_driver_config const &c = cfgs[r];
        double const L[3] = {c.box[0], c.box[4], c.box[8]};
        for (int a = 0; a < c.n_atoms; ++a) {
            double const *p = c.positions + 3 * a;
            double const u[3] = {p[0] / L[0], p[1] / L[1], p[2] / L[2]};
            size_t const i = static_cast<size_t>(begin[r] + a);
            crd[i] = make_double4(u[0] - nint_host(u[0]), u[1] - nint_host(u[1]),
                                  u[2] - nint_host(u[2]), static_cast<double>(c.types[a]));
            rep_of[i] = r;
            for (int k = 0; k < 3; ++k) {
                vel[static_cast<size_t>(k) * np + i] = c.velocities[3 * a + k];
                pos0[static_cast<size_t>(p0off + 3 * a + k)] = p[k];
            }
        }
        // padding slots up to the next replica's block: no atom
        int const end = r + 1 < n_rep ? begin[r + 1] : np;
        for (int i = begin[r] + c.n_atoms; i < end; ++i) {
            crd[i] = make_double4(0., 0., 0., 0.);
            rep_of[i] = -1;
            for (int k = 0; k < 3; ++k)
                vel[static_cast<size_t>(k) * np + i] = 0.;
        }
        p0off += 3L * c.n_atoms;
    }

    auto *d = new mdelast_driver_s();
    d->device = c0.device;
    if (cudaDeviceGetAttribute(&d->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                               d->device) != cudaSuccess)
        d->smem_optin = 48 * 1024;
    if (char const *e = std::getenv("MDELAST_CELL_STAGING"))
        d->cell_staging = std::atoi(e) != 0;
    auto bail = [&](int rc) {
        delete d;
        return rc;
    };
#define TRY(x)                                                                                \
    do {                                                                                      \
        int rc_ = (x);                                                                        \
        if (rc_)                                                                              \
            return bail(rc_);                                                                 \
    } while (0)
    if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(MDELAST_ERR_CUDA, "stream creation failed"));
    d->n_rep = n_rep;
    d->rep_begin = begin;
    d->rep_count = count;
    d->N = static_cast<int>(n_total);
    d->ntypes = nt;
    d->npot = npot;
    d->n_pad = np;
    d->n_blocks = np / kBlock;
    d->neighbors = c0.neighbors != 0;
    d->r_skin = c0.r_skin;
    mdelast_pair const *p0 = c0.pair[0];
    double const rcut = p0->rcut;
    d->r_list = d->neighbors ? rcut * c0.r_skin : rcut;

    // ---- tables: r-table bundles and embedding tables. Per interval and function, the 6
    // quintic coefficients, or for "bspline" the 12 coefficients of the three cubics
    int const interp = p0->interpolation;
    bool const bsp = interp == MDELAST_BSPLINE;
    size_t const kF = bsp ? 12 : 6;
    auto fun = [&](mdelast::QuinticTable const &q, int k) {
        return (bsp ? q.cub.data() : q.coef.data()) + kF * static_cast<size_t>(k);
    };
    int const nri = p0->table.n;
    std::vector<double> rb(static_cast<size_t>(npot) * nri * 3 * kF, 0.);
    for (int b = 0; b < nt; ++b)
        for (int a = 0; a <= b; ++a) {
            int const s = b * (b + 1) / 2 + a;
            for (int k = 0; k < nri; ++k) {
                double *o = rb.data() + (static_cast<size_t>(s) * nri + k) * 3 * kF;
                std::memcpy(o, fun(c0.pair[s]->table, k), kF * sizeof(double));
                if (c0.n_eam) {
                    std::memcpy(o + kF, fun(c0.eam[a]->rho, k), kF * sizeof(double));
                    std::memcpy(o + 2 * kF, fun(c0.eam[b]->rho, k), kF * sizeof(double));
                }
            }
        }
    int const nfi = c0.n_eam ? c0.eam[0]->F.n : 1;
    std::vector<double> Ft(static_cast<size_t>(nt) * nfi * kF, 0.);
    for (int t = 0; t < c0.n_eam; ++t)
        for (int k = 0; k < nfi; ++k)
            std::memcpy(Ft.data() + (static_cast<size_t>(t) * nfi + k) * kF,
                        fun(c0.eam[t]->F, k), sizeof(double) * kF);
    TRY(dalloc(&d->d_rb, rb.size()));
    TRY(dalloc(&d->d_Ft, Ft.size()));
    if (cudaMemcpy(d->d_rb, rb.data(), sizeof(double) * rb.size(), cudaMemcpyHostToDevice) ||
        cudaMemcpy(d->d_Ft, Ft.data(), sizeof(double) * Ft.size(), cudaMemcpyHostToDevice))
        return bail(fail(MDELAST_ERR_CUDA, "table upload failed"));
    TablesView &T = d->T;
    T.rb = d->d_rb;
    T.nri = nri;
    T.npot = npot;
    T.inv_hr = p0->table.inv_h;
    T.inv_hr2 = p0->table.inv_h2;
    T.Ft = d->d_Ft;
    T.nfi = nfi;
    T.ntypes = nt;
    T.inv_hf = c0.n_eam ? c0.eam[0]->F.inv_h : 1.;
    T.inv_hf2 = c0.n_eam ? c0.eam[0]->F.inv_h2 : 1.;
    T.has_eam = c0.n_eam > 0;
    T.interp = interp;
    T.r_cut_sq = rcut * rcut;
    for (int s = 0; s < npot; ++s) {
        T.pot_rcut[s] = c0.pair[s]->rcut;
        T.pot_rmin[s] = c0.pair[s]->rmin_fatal;
    }
    for (int t = 0; t < nt; ++t) {
        T.eam_rcut[t] = c0.n_eam ? c0.eam[t]->rcut : 0.;
        T.rhomax[t] = c0.n_eam ? c0.eam[t]->rhomax_fatal : 0.;
        T.mass[t] = c0.mass[t];
    }
    {
        double const rc64 = std::sqrt(T.r_cut_sq);
        T.uc64 = 1;
        for (int s = 0; s < npot; ++s)
            T.uc64 &= T.pot_rcut[s] >= rc64;
        if (T.has_eam)
            for (int t = 0; t < nt; ++t)
                T.uc64 &= T.eam_rcut[t] >= rc64;
    }
    d->precision = c0.precision;
    if (c0.precision == MDELAST_PRECISION_MIXED) {
        // The r tables in FP32, angstrom / eV (phi) and angstrom^-3 (rho): per type pair
        // and interval a bundle of phi_ab, rho_a, rho_b; per type and interval rho. Quintic
        // coefficients carry the function's unit (derivatives come with 1/h in angstrom);
        // the bspline cubics of f' and f'' carry one and two more 1/length.
        size_t const kFf = bsp ? 12 : 6, kFb = bsp ? 12 : 6, kB = 3 * kFb;
        double const a3 = kAng * kAng * kAng;
        auto pack = [&](const double *src, double unit, float *dst) {
            for (size_t c = 0; c < kF; ++c) {
                double f = unit;
                for (size_t q = 0; bsp && q < c / 4; ++q) // 0 f, 1 f', 2 f''
                    f *= kAng;
                dst[c] = static_cast<float>(src[c] * f);
            }
        };
        std::vector<float> rbf(static_cast<size_t>(npot) * nri * kB, 0.f);
        std::vector<float> rrf(static_cast<size_t>(nt) * nri * kFf, 0.f);
        for (int b = 0; b < nt; ++b)
            for (int a = 0; a <= b; ++a) {
                int const s = b * (b + 1) / 2 + a;
                for (int k = 0; k < nri; ++k) {
                    float *o = rbf.data() + (static_cast<size_t>(s) * nri + k) * kB;
                    pack(fun(c0.pair[s]->table, k), 1. / kEv, o);
                    if (c0.n_eam) {
                        pack(fun(c0.eam[a]->rho, k), a3, o + kFb);
                        pack(fun(c0.eam[b]->rho, k), a3, o + 2 * kFb);
                    }
                }
            }
        for (int t = 0; t < c0.n_eam; ++t)
            for (int k = 0; k < nri; ++k)
                pack(fun(c0.eam[t]->rho, k), a3,
                     rrf.data() + (static_cast<size_t>(t) * nri + k) * kFf);
        TRY(dalloc(&d->d_rbf, rbf.size()));
        TRY(dalloc(&d->d_rrf, rrf.size()));
        if (cudaMemcpy(d->d_rbf, rbf.data(), sizeof(float) * rbf.size(), cudaMemcpyHostToDevice) ||
            cudaMemcpy(d->d_rrf, rrf.data(), sizeof(float) * rrf.size(), cudaMemcpyHostToDevice))
            return bail(fail(MDELAST_ERR_CUDA, "table upload failed"));
        T.rbf = d->d_rbf;
        T.rrf = d->d_rrf;
        // The staged copy of the force pass: every phi_ab, then every rho_a, over the top
        // intervals of the r grid (those below r_cut, as many as kStageBudget holds), the
        // same FP32 values as the bundles. Quintic EAM tables only.
        if (!bsp && c0.n_eam) {
            int const n_fun = npot + nt;
            double rc_max = 0.;
            for (int q = 0; q < npot; ++q)
                rc_max = std::max(rc_max, T.pot_rcut[q]);
            for (int q = 0; q < nt; ++q)
                rc_max = std::max(rc_max, T.eam_rcut[q]);
            long const k_hi = std::min<long>(
                nri, static_cast<long>(std::floor(rc_max / kAng * (T.inv_hr * kAng))) + 2);
            long const fit = kStageBudget / (static_cast<long>(n_fun) * 24);
            long const n_st = std::min(k_hi, fit);
            if (n_st >= 16) {
                long const lo = k_hi - n_st;
                size_t const nfl = static_cast<size_t>(n_fun) * n_st * 6;
                std::vector<float> stf((nfl + 3) / 4 * 4, 0.f);
                for (int q = 0; q < n_fun; ++q)
                    for (long k = 0; k < n_st; ++k) {
                        float *o = stf.data() + (static_cast<size_t>(q) * n_st + k) * 6;
                        if (q < npot)
                            pack(fun(c0.pair[q]->table, static_cast<int>(lo + k)), 1. / kEv, o);
                        else
                            pack(fun(c0.eam[q - npot]->rho, static_cast<int>(lo + k)), a3, o);
                    }
                TRY(dalloc(&d->d_stf, stf.size()));
                if (cudaMemcpy(d->d_stf, stf.data(), sizeof(float) * stf.size(),
                               cudaMemcpyHostToDevice))
                    return bail(fail(MDELAST_ERR_CUDA, "table upload failed"));
                T.stf = d->d_stf;
                T.st_lo = static_cast<int>(lo);
                T.st_n = static_cast<int>(n_st);
                T.st_bytes = static_cast<int>(sizeof(float) * stf.size());
                // the kernels' limit is the budget, not this copy's size: another driver
                // in the process may stage a larger copy
                if (cudaError_t e = prepare_force_mx_staged(static_cast<int>(kStageBudget)))
                    return bail(fail(MDELAST_ERR_CUDA, "staged kernels: %s", cudaGetErrorString(e)));
            }
        }
        T.finv_hr = static_cast<float>(T.inv_hr * kAng);
        T.finv_hr2 = static_cast<float>(T.inv_hr2 * kAng * kAng);
        T.fr_cut_sq = static_cast<float>((rcut / kAng) * (rcut / kAng));
        for (int s = 0; s < npot; ++s) {
            T.fpot_rcut[s] = static_cast<float>(T.pot_rcut[s] / kAng);
            T.fpot_rmin[s] = static_cast<float>(T.pot_rmin[s] / kAng);
        }
        for (int t = 0; t < nt; ++t)
            T.feam_rcut[t] = static_cast<float>(T.eam_rcut[t] / kAng);
        float const rcf = static_cast<float>(rcut / kAng);
        T.fuc = 1;
        for (int s = 0; s < npot; ++s)
            T.fuc &= T.fpot_rcut[s] >= rcf;
        if (T.has_eam)
            for (int t = 0; t < nt; ++t)
                T.fuc &= T.feam_rcut[t] >= rcf;
    }

    // ---- g(r) bins of each replica (md_driver.cpp:41): drg = rg[1] - rg[0],
    // rmaxg = rg[n - 1] + drg / 2
    {
        long off = 0;
        size_t max_slots = 0;
        std::vector<double> rg_all;
        for (int r = 0; r < n_rep; ++r) {
            mdelast_driver_config const &c = cfgs[r];
            d->gr_off.push_back(off);
            d->gr_n.push_back(c.n_rg);
            d->gr_drg.push_back(c.rg[1] - c.rg[0]);
            d->gr_rmax.push_back(c.rg[c.n_rg - 1] + 0.5 * (c.rg[1] - c.rg[0]));
            rg_all.insert(rg_all.end(), c.rg, c.rg + c.n_rg);
            off += c.n_rg;
            max_slots = std::max(max_slots, gr_count_slots(c.n_rg, nt));
        }
        TRY(dalloc(&d->d_rg, rg_all.size()));
        TRY(dalloc(&d->d_gr, rg_all.size()));
        TRY(dalloc(&d->d_grp, rg_all.size() * static_cast<size_t>(npot)));
        TRY(dalloc(&d->d_gr_counts, max_slots));
        TRY(dalloc(&d->d_gr_ntype, static_cast<size_t>(nt)));
        if (cudaMemcpy(d->d_rg, rg_all.data(), sizeof(double) * rg_all.size(),
                       cudaMemcpyHostToDevice))
            return bail(fail(MDELAST_ERR_CUDA, "rg upload failed"));
    }

    // ---- replica states
    std::vector<Replica> R(static_cast<size_t>(n_rep));
    std::vector<Replica *> reps;
    for (int r = 0; r < n_rep; ++r) {
        mdelast_driver_config const &c = cfgs[r];
        Replica &x = R[static_cast<size_t>(r)];
        std::memset(&x, 0, sizeof(Replica));
        x.atom_begin = begin[r];
        x.n_atoms = c.n_atoms;
        x.block_begin = begin[r] / kBlock;
        x.n_blocks = (c.n_atoms + kTile - 1) / kTile * kTile / kBlock;
        x.ensemble = c.ensemble;
        x.coupling = c.coupling;
        x.Nf = c.Nf;
        x.alpha = 1. + 3. / c.Nf;
        x.dt = c.dt;
        x.fatal_conservation = c.fatal_conservation;
        x.mass0 = c.mass[0];
        x.baro_P = c.baro_P;
        x.baro_w = c.baro_w;
        for (int a = 0; a < 3; ++a)
            x.h0[a] = x.h[a] = x.h_pos[a] = c.box[4 * a];
        x.eps = 0.;
        x.p_eps = c.baro_p_eps;
        x.vscale = 1.;
        x.acc.n_atoms = c.n_atoms;
        set_chain(x.th, c.thermo_T, c.thermo_nchain, c.thermo_q, c.thermo_p_eta, c.thermo_Nf);
        set_chain(x.bth, c.baro_thermo_T, c.baro_nchain, c.baro_q, c.baro_p_eta, c.baro_Nf);
        reps.push_back(&x);
    }
    d->tpa_d = d->tpa_f = default_tpa(static_cast<int>(std::min<long>(n_total, 1L << 30)));
    std::vector<int> dmap, fmap;
    d->grid_d = deal_blocks(reps, d->tpa_d, true, dmap);
    d->grid_f = deal_blocks(reps, d->tpa_f, false, fmap);
    TRY(dalloc(&d->d_dblk_rep, dmap.size()));
    TRY(dalloc(&d->d_fblk_rep, fmap.size()));
    d->cap_dmap = dmap.size();
    d->cap_fmap = fmap.size();
    TRY(dalloc(&d->d_rep, static_cast<size_t>(n_rep)));
    if (cudaMemcpy(d->d_rep, R.data(), sizeof(Replica) * n_rep, cudaMemcpyHostToDevice) ||
        cudaMemcpy(d->d_dblk_rep, dmap.data(), sizeof(int) * dmap.size(), cudaMemcpyHostToDevice) ||
        cudaMemcpy(d->d_fblk_rep, fmap.data(), sizeof(int) * fmap.size(), cudaMemcpyHostToDevice))
        return bail(fail(MDELAST_ERR_CUDA, "state upload failed"));

    // ---- atoms
    TRY(dalloc(&d->d_rep_of, np));
    TRY(dalloc(&d->d_crd, np));
    TRY(dalloc(&d->d_vel, 3 * static_cast<size_t>(np)));
    TRY(dalloc(&d->d_frc, 3 * static_cast<size_t>(np)));
    TRY(dalloc(&d->d_rho, np));
    TRY(dalloc(&d->d_Fe, np));
    TRY(dalloc(&d->d_epot, np));
    TRY(dalloc(&d->d_dF2, np));
    if (c0.precision == MDELAST_PRECISION_MIXED) {
        TRY(dalloc(&d->d_posf, np));
        TRY(dalloc(&d->d_dF2f, np));
    }
    TRY(dalloc(&d->d_nup, np));
    TRY(dalloc(&d->d_ndn, np));
    TRY(dalloc(&d->d_pd, static_cast<size_t>(d->grid_d) * D_NSUM));
    TRY(dalloc(&d->d_pf, static_cast<size_t>(d->grid_f) * F_NSUM));
    d->cap_pd = static_cast<size_t>(d->grid_d) * D_NSUM;
    d->cap_pf = static_cast<size_t>(d->grid_f) * F_NSUM;
    int max_chunks = 1;
    for (Replica const *x : reps)
        max_chunks = std::max(max_chunks, (std::max(x->dblk_n, x->fblk_n) + kChunk - 1) / kChunk);
    TRY(dalloc(&d->d_red, static_cast<size_t>(n_rep) * max_chunks * 64));
    d->cap_red = static_cast<size_t>(n_rep) * max_chunks * 64;
    TRY(dalloc(&d->d_max_count, 2));
    TRY(dalloc(&d->d_halt, 1));
    TRY(dalloc(&d->d_pos0, 3 * static_cast<size_t>(n_total)));
    int max_n = 0;
    for (int r = 0; r < n_rep; ++r)
        max_n = std::max(max_n, count[r]);
    TRY(dalloc(&d->d_out, 3 * static_cast<size_t>(max_n)));
    d->pos0_off.assign(static_cast<size_t>(n_rep), 0);
    for (int r = 1; r < n_rep; ++r)
        d->pos0_off[r] = d->pos0_off[r - 1] + 3L * count[r - 1];
    if (cudaMemcpyAsync(d->d_rep_of, rep_of, b_rep, cudaMemcpyHostToDevice, d->stream) ||
        cudaMemcpyAsync(d->d_crd, crd, b_crd, cudaMemcpyHostToDevice, d->stream) ||
        cudaMemcpyAsync(d->d_vel, vel, b_vel, cudaMemcpyHostToDevice, d->stream) ||
        cudaMemcpyAsync(d->d_pos0, pos0, b_pos0, cudaMemcpyHostToDevice, d->stream) ||
        cudaStreamSynchronize(d->stream))
        return bail(fail(MDELAST_ERR_CUDA, "atom upload failed"));
    stage_lock.unlock(); // the staging is free for the next creation
    if (cudaMallocHost(&d->h_obs, sizeof(mdelast_observables) * n_rep) ||
        cudaEventCreateWithFlags(&d->ev_step, cudaEventDisableTiming))
        return bail(fail(MDELAST_ERR_CUDA, "host staging allocation failed"));

    AtomsView &A = d->A;
    A.n_pad = np;
    A.n_rep = n_rep;
    A.rep = d->d_rep;
    A.rep_of = d->d_rep_of;
    A.crd = d->d_crd;
    A.vel = d->d_vel;
    A.frc = d->d_frc;
    A.rho = d->d_rho;
    A.Fe = d->d_Fe;
    A.epot = d->d_epot;
    A.dF2 = d->d_dF2;
    A.posf = d->d_posf;
    A.dF2f = d->d_dF2f;
    A.n_up = d->d_nup;
    A.n_dn = d->d_ndn;
    A.pd = d->d_pd;
    A.pf = d->d_pf;
    A.red = d->d_red;
    A.max_chunks = max_chunks;
    A.dblk_rep = d->d_dblk_rep;
    A.fblk_rep = d->d_fblk_rep;
    A.max_count = d->d_max_count;
    A.halt = d->d_halt;
    TRY(d->alloc_ring(MDELAST_DEFAULT_SAMPLE_RING));
    if (d->neighbors) // md_driver.cpp:42: pow<2>(pot[0]->rcut * r_skin)
        A.r_list_sq = (rcut * c0.r_skin) * (rcut * c0.r_skin);
    else
        A.r_list_sq = rcut * rcut;

    // neighbour capacity from the densest replica: 1.5 x its mean count + 32
    int maxn = 4;
    for (int r = 0; r < n_rep; ++r) {
        mdelast_driver_config const &c = cfgs[r];
        double const vol = c.box[0] * (c.box[4] * c.box[8]);
        double const mean = 4. / 3. * M_PI * std::pow(d->r_list, 3) * c.n_atoms / vol;
        double const h = list_headroom();
        int m = static_cast<int>((1. + h) * std::min(mean, static_cast<double>(c.n_atoms))) +
                (h > 0. ? 32 : 0);
        m = std::min((m + 3) / 4 * 4, (c.n_atoms + 3) / 4 * 4);
        maxn = std::max(maxn, m);
    }
    TRY(d->alloc_list(maxn));
    std::vector<double> boxes;
    for (int r = 0; r < n_rep; ++r)
        for (int a = 0; a < 3; ++a)
            boxes.push_back(cfgs[r].box[4 * a]);
    TRY(d->configure_cells(boxes));

    // ---- the constructor's force call and thermodynamics (md_driver.cpp:112-118)
    TRY(d->build_list_checked());
    if (d->A.posf)
        k_posf<<<np / kBlock, kBlock, 0, d->stream>>>(d->A);
    {
        double f = 1.06; // pairs within 1.06 r_cut; MDELAST_PAIR_LIST=0 reads the full list
        if (char const *e = std::getenv("MDELAST_PAIR_LIST"))
            f = std::atof(e);
        d->rcut0 = rcut;
        TRY(d->set_pair_list(f));
    }
    d->pass_density(true, d->stream);
    d->pass_force(true, false, d->stream);
    d->post(POST_INIT, 1, d->stream);
    if (cudaGetLastError() != cudaSuccess)
        return bail(fail(MDELAST_ERR_CUDA, "kernel launch failed"));
    if (cudaMemcpy2DAsync(d->h_obs, sizeof(mdelast_observables),
                          reinterpret_cast<char *>(d->d_rep) + offsetof(Replica, obs),
                          sizeof(Replica), sizeof(mdelast_observables), d->n_rep,
                          cudaMemcpyDeviceToHost, d->stream) ||
        cudaStreamSynchronize(d->stream))
        return bail(fail(MDELAST_ERR_CUDA, "constructor force call failed: %s",
                         cudaGetErrorString(cudaGetLastError())));
    d->obs_valid = true;
    TRY(d->check_status());
#undef TRY
    *out = d;
    return MDELAST_OK;
}

extern "C" {

int mdelast_driver_create(const mdelast_driver_config *cfg, mdelast_driver **out) {
    return create_system(cfg, 1, out);
}

void mdelast_driver_destroy(mdelast_driver *d) { delete d; }

int mdelast_driver_integrate(mdelast_driver *d, int32_t n_steps) {
    clear_error();
    if (!d || n_steps < 0)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    if (d->dead)
        return d->check_status();
    CK(cudaSetDevice(d->device));
    return d->launch_steps(n_steps, -1, -1);
}

int mdelast_driver_run(mdelast_driver *d, int32_t n_steps, int32_t rebuild_every,
                       int32_t sample_every, float *device_ms) {
    clear_error();
    if (!d || n_steps < 0)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    if (d->neighbors && rebuild_every > 0) { // cell geometry for the current box
        if (int rc = d->configure_cells(d->current_boxes()))
            return rc;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (device_ms) {
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        CK(cudaEventRecord(e0, d->stream));
    }
    int rc = d->launch_steps(n_steps, d->neighbors ? rebuild_every : 0, sample_every);
    if (device_ms && !rc) {
        cudaEventRecord(e1, d->stream);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(device_ms, e0, e1);
        if (e != cudaSuccess)
            rc = fail(MDELAST_ERR_CUDA, "step timing: %s", cudaGetErrorString(e));
    }
    if (e0)
        cudaEventDestroy(e0);
    if (e1)
        cudaEventDestroy(e1);
    return rc;
}

int mdelast_driver_kernel_times(mdelast_driver *d, int32_t n_steps, double *ms_out) {
    clear_error();
    if (!d || n_steps < 1 || !ms_out)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    std::vector<cudaEvent_t> ev(8);
    for (auto &e : ev)
        CK(cudaEventCreate(&e));
    double acc[MDELAST_N_KERNEL_TIMES] = {0, 0, 0, 0, 0, 0};
    int const grid = d->n_pad / kBlock;
    cudaStream_t s = d->stream;
    int rc = MDELAST_OK;
    for (int step = 0; step < n_steps && !rc; ++step) {
        cudaEventRecord(ev[0], s);
        if (d->neighbors || step == 0)
            rc = d->enqueue_rebuild();
        cudaEventRecord(ev[1], s);
        k_pre<<<d->n_rep, 64, 0, s>>>(d->A);
        cudaEventRecord(ev[2], s);
        k_kick_drift<<<grid, kBlock, 0, s>>>(d->A, d->T);
        cudaEventRecord(ev[3], s);
        d->refresh_pair_list(s);
        cudaEventRecord(ev[7], s);
        d->pass_density(true, s);
        cudaEventRecord(ev[4], s);
        d->pass_force(true, true, s);
        cudaEventRecord(ev[5], s);
        d->post(POST_STEP, 1, s);
        cudaEventRecord(ev[6], s);
        cudaError_t e = cudaEventSynchronize(ev[6]);
        if (e != cudaSuccess) {
            rc = fail(MDELAST_ERR_CUDA, "kernel timing: %s", cudaGetErrorString(e));
            break;
        }
        // pre, kick+drift, density, force, closing scalar work, list build + pair-list
        // refresh
        float t[6], u = 0.f;
        cudaEventElapsedTime(&t[0], ev[1], ev[2]);
        cudaEventElapsedTime(&t[1], ev[2], ev[3]);
        cudaEventElapsedTime(&t[2], ev[7], ev[4]);
        cudaEventElapsedTime(&t[3], ev[4], ev[5]);
        cudaEventElapsedTime(&t[4], ev[5], ev[6]);
        cudaEventElapsedTime(&t[5], ev[0], ev[1]);
        cudaEventElapsedTime(&u, ev[3], ev[7]);
        t[5] += u;
        for (int k = 0; k < 6; ++k)
            acc[k] += t[k];
        ++d->host_cycle;
    }
    for (auto &e : ev)
        cudaEventDestroy(e);
    for (int k = 0; k < MDELAST_N_KERNEL_TIMES; ++k)
        ms_out[k] = acc[k] / n_steps;
    d->stepped = true;
    CK(cudaMemcpy2D(d->h_obs, sizeof(mdelast_observables),
                    reinterpret_cast<char *>(d->d_rep) + offsetof(Replica, obs), sizeof(Replica),
                    sizeof(mdelast_observables), d->n_rep, cudaMemcpyDeviceToHost));
    d->obs_valid = true;
    if (rc)
        return rc;
    return d->check_status();
}

int mdelast_driver_calculate_neighbors(mdelast_driver *d) {
    clear_error();
    if (!d)
        return fail(MDELAST_ERR_ARGUMENT, "null driver");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    if (!d->neighbors) // the reference writes into empty point/neighbors storage
        return fail(MDELAST_ERR_UNSUPPORTED,
                    "calculate_neighbors() needs a driver created with neighbors=True");
    if (int rc = d->configure_cells(d->current_boxes()))
        return rc;
    return d->build_list_checked();
}

int mdelast_driver_set_sample_observables(mdelast_driver *d, int32_t flag) {
    if (!d)
        return fail(MDELAST_ERR_ARGUMENT, "null driver");
    d->sample = flag != 0;
    return MDELAST_OK;
}

int mdelast_driver_get_sample_observables(const mdelast_driver *d, int32_t *flag) {
    if (!d || !flag)
        return fail(MDELAST_ERR_ARGUMENT, "null argument");
    *flag = d->sample;
    return MDELAST_OK;
}

int mdelast_driver_synchronize(mdelast_driver *d) {
    clear_error();
    if (!d)
        return fail(MDELAST_ERR_ARGUMENT, "null driver");
    CK(cudaSetDevice(d->device));
    CK(cudaStreamSynchronize(d->stream));
    return d->wait_step();
}

} // extern "C"

// Readouts of replica r (r = 0 for a single driver).
static int get_observables_r(mdelast_driver *d, int r, mdelast_observables *out) {
    clear_error();
    if (!d || !out || r < 0 || r >= d->n_rep)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    CK(cudaSetDevice(d->device));
    int const rc = d->wait_step();
    *out = d->h_obs[r];
    return rc;
}

static int get_atoms_r(mdelast_driver *d, int r, int32_t field, double *out) {
    clear_error();
    if (!d || !out || field < 0 || field > MDELAST_ATOM_EKIN || r < 0 || r >= d->n_rep)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    int const N = d->rep_count[r];
    k_readout<<<(N + 255) / 256, 256, 0, d->stream>>>(d->A, d->T, r, field, d->d_out,
                                                      d->d_pos0 + d->pos0_off[r],
                                                      d->stepped ? 1 : 0);
    CK(cudaGetLastError());
    size_t const n = field <= MDELAST_ATOM_FORCES ? 3 * static_cast<size_t>(N) : N;
    CK(cudaMemcpyAsync(out, d->d_out, sizeof(double) * n, cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    return MDELAST_OK;
}

static int get_chain_r(mdelast_driver *d, int r, int32_t which, double *q, double *p_eta,
                       double *eta, int32_t *nchain) {
    clear_error();
    if (!d || (which != 0 && which != 1) || r < 0 || r >= d->n_rep)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    Chain ch;
    size_t const off = static_cast<size_t>(r) * sizeof(Replica) +
                       (which == 0 ? offsetof(Replica, th) : offsetof(Replica, bth));
    CK(cudaMemcpy(&ch, reinterpret_cast<char *>(d->d_rep) + off, sizeof(Chain),
                  cudaMemcpyDeviceToHost));
    for (int j = 0; j < ch.n; ++j) {
        if (q)
            q[j] = ch.q[j];
        if (p_eta)
            p_eta[j] = ch.p_eta[j];
        if (eta)
            eta[j] = ch.eta[j];
    }
    if (nchain)
        *nchain = ch.n;
    return MDELAST_OK;
}

static int get_neighbors_r(mdelast_driver *d, int r, int32_t *point, int32_t *neighbors,
                           int64_t cap, int64_t *n_entries) {
    clear_error();
    if (!d || !point || r < 0 || r >= d->n_rep)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    if (!d->neighbors)
        return fail(MDELAST_ERR_UNSUPPORTED, "neighbour lists are disabled for this driver");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    int const N = d->rep_count[r];
    if (d->tmp_i_cap < static_cast<size_t>(N) + 1) {
        dfree(d->d_tmp_i);
        if (int rc = dalloc(&d->d_tmp_i, static_cast<size_t>(N) + 1))
            return rc;
        d->tmp_i_cap = static_cast<size_t>(N) + 1;
    }
    k_half_list_counts<<<(N + 255) / 256, 256, 0, d->stream>>>(d->A, r, d->d_tmp_i);
    std::vector<int> cnt(static_cast<size_t>(N));
    CK(cudaMemcpyAsync(cnt.data(), d->d_tmp_i, sizeof(int) * N, cudaMemcpyDeviceToHost,
                       d->stream));
    CK(cudaStreamSynchronize(d->stream));
    int64_t total = 0;
    for (int i = 0; i < N; ++i) {
        point[i] = static_cast<int32_t>(total);
        total += cnt[static_cast<size_t>(i)];
    }
    point[N] = static_cast<int32_t>(total);
    if (n_entries)
        *n_entries = total;
    if (!neighbors || cap <= 0)
        return MDELAST_OK;
    int *d_point = nullptr, *d_list = nullptr;
    if (int rc = dalloc(&d_point, static_cast<size_t>(N) + 1))
        return rc;
    if (int rc = dalloc(&d_list, static_cast<size_t>(std::max<int64_t>(total, 1)))) {
        dfree(d_point);
        return rc;
    }
    cudaError_t e = cudaMemcpy(d_point, point, sizeof(int) * (N + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_half_list_fill<<<(N + 255) / 256, 256, 0, d->stream>>>(d->A, r, d_point, d_list);
        e = cudaMemcpyAsync(neighbors, d_list,
                            sizeof(int) * static_cast<size_t>(std::min(total, cap)),
                            cudaMemcpyDeviceToHost, d->stream);
    }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(d->stream);
    dfree(d_point);
    dfree(d_list);
    if (e != cudaSuccess)
        return fail(MDELAST_ERR_CUDA, "neighbour readout: %s", cudaGetErrorString(e));
    return MDELAST_OK;
}

// md_driver.cpp:732-862 on the device: counts and normalises on the driver's stream after
// the last step launched; get_gr_r waits for it.
static int pair_correlation_r(mdelast_driver *d, int r, int32_t mode) {
    clear_error();
    if (!d || r < 0 || r >= d->n_rep || mode < 0 || mode > 2)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    if (!gr_atoms_fit(d->rep_count[r]))
        return fail(MDELAST_ERR_CAPACITY,
                    "g(r) of %d atoms needs more than 2^31 - 1 blocks of 128-atom tile pairs",
                    d->rep_count[r]);
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    GrArgs g{};
    g.crd = d->d_crd + d->rep_begin[r];
    g.rep = d->d_rep + r;
    g.n = d->rep_count[r];
    g.ntypes = d->ntypes;
    g.n_rg = d->gr_n[r];
    g.mode = mode;
    g.rg = d->d_rg + d->gr_off[r];
    g.drg = d->gr_drg[r];
    g.rmaxg = d->gr_rmax[r];
    g.counts = d->d_gr_counts;
    g.n_per_type = d->d_gr_ntype;
    g.gr = d->d_gr + d->gr_off[r];
    g.gr_partial = d->d_grp + static_cast<size_t>(d->npot) * d->gr_off[r];
    CK(gr_enqueue(g, d->stream));
    return MDELAST_OK;
}

static int get_gr_r(mdelast_driver *d, int r, double *gr, double *gr_partial) {
    clear_error();
    if (!d || r < 0 || r >= d->n_rep)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    CK(cudaSetDevice(d->device));
    size_t const n = static_cast<size_t>(d->gr_n[r]);
    if (gr)
        CK(cudaMemcpyAsync(gr, d->d_gr + d->gr_off[r], sizeof(double) * n,
                           cudaMemcpyDeviceToHost, d->stream));
    if (gr_partial)
        CK(cudaMemcpyAsync(gr_partial, d->d_grp + static_cast<size_t>(d->npot) * d->gr_off[r],
                           sizeof(double) * n * d->npot, cudaMemcpyDeviceToHost, d->stream));
    CK(cudaStreamSynchronize(d->stream));
    return MDELAST_OK;
}

// Records of replica r written since its last drain (molecular_dynamics.py:1218-1238).
static int drain_samples_r(mdelast_driver *d, int r, mdelast_sample *out, int64_t cap,
                           int64_t *n_out, int64_t *n_lost) {
    clear_error();
    if (!d || r < 0 || r >= d->n_rep || cap < 0 || (cap > 0 && !out))
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    double written_d = 0.;
    CK(cudaMemcpy(&written_d,
                  reinterpret_cast<char *>(d->d_rep + r) + offsetof(Replica, n_samples),
                  sizeof(double), cudaMemcpyDeviceToHost));
    long long const written = static_cast<long long>(written_d);
    long long const ringc = d->A.ring_cap;
    long long &done = d->drained[static_cast<size_t>(r)];
    long long const first = ringc > 0 ? std::max(done, written - ringc) : written;
    long long const lost = first - done;
    long long const count = std::min<long long>(written - first, cap);
    mdelast_sample const *base = d->d_ring + static_cast<size_t>(r) * (ringc > 0 ? ringc : 0);
    long long k = 0;
    while (k < count) { // at most two contiguous pieces of the ring
        long long const slot = (first + k) % ringc;
        long long const len = std::min(count - k, ringc - slot);
        CK(cudaMemcpyAsync(out + k, base + slot, sizeof(mdelast_sample) * len,
                           cudaMemcpyDeviceToHost, d->stream));
        k += len;
    }
    CK(cudaStreamSynchronize(d->stream));
    done = first + count;
    if (n_out)
        *n_out = count;
    if (n_lost)
        *n_lost = lost;
    return MDELAST_OK;
}

static int get_fluct_r(mdelast_driver *d, int r, mdelast_fluct *out) {
    clear_error();
    if (!d || !out || r < 0 || r >= d->n_rep)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    CK(cudaMemcpy(out, reinterpret_cast<char *>(d->d_rep + r) + offsetof(Replica, acc),
                  sizeof(mdelast_fluct), cudaMemcpyDeviceToHost));
    return MDELAST_OK;
}

extern "C" {

int mdelast_driver_autotune(mdelast_driver *d, int32_t n_repeat, int32_t *choice,
                            double *ms_out) {
    clear_error();
    if (!d || n_repeat < 1)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    int const tpas[4] = {1, 4, 8, 16};
    int const targets[4] = {148 * 8, 148 * 16, 148 * 32, 148 * 64};
    double best_d = 1e300, best_f = 1e300;
    int bd[2] = {d->tpa_d, d->target_d}, bf[3] = {d->tpa_f, d->target_f, d->stage_f ? 1 : 0};
    for (int tp : tpas)
        for (int tg : targets) {
            if (int rc = d->set_launch(tp, tp, tg, tg, 0))
                return rc;
            double md = 0., mf = 0.;
            if (int rc = d->time_passes(n_repeat, d->sample, &md, &mf))
                return rc;
            if (md < best_d) {
                best_d = md;
                bd[0] = tp;
                bd[1] = tg;
            }
            if (mf < best_f) {
                best_f = mf;
                bf[0] = tp;
                bf[1] = tg;
                bf[2] = 0;
            }
        }
    // the staged force pass: one 512-thread block per SM, one to four waves
    if (d->staging_available())
        for (int tp : {4, 8, 16})
            for (int tg : {148, 148 * 2, 148 * 4}) {
                if (int rc = d->set_launch(bd[0], tp, bd[1], tg, 1))
                    return rc;
                double md = 0., mf = 0.;
                if (int rc = d->time_passes(n_repeat, d->sample, &md, &mf))
                    return rc;
                if (mf < best_f) {
                    best_f = mf;
                    bf[0] = tp;
                    bf[1] = tg;
                    bf[2] = 1;
                }
            }
    if (int rc = d->set_launch(bd[0], bf[0], bd[1], bf[1], bf[2]))
        return rc;
    // recompute the per-atom state with the chosen shapes (positions are unchanged)
    double md = 0., mf = 0.;
    if (int rc = d->time_passes(1, 1, &md, &mf))
        return rc;
    if (choice) {
        choice[0] = bd[0];
        choice[1] = bf[0];
        choice[2] = bd[1];
        choice[3] = bf[1];
    }
    if (ms_out) {
        ms_out[0] = best_d;
        ms_out[1] = best_f;
    }
    return MDELAST_OK;
}

int mdelast_driver_autotune_steps(mdelast_driver *d, int32_t n_steps, int32_t rebuild_every,
                                  int32_t *choice, double *ms_out) {
    clear_error();
    if (!d || n_steps < 1)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    if (d->neighbors && rebuild_every > 0)
        if (int rc = d->configure_cells(d->current_boxes()))
            return rc;
    int c[4];
    double ms[2];
    if (int rc = d->tune_on_steps(n_steps, rebuild_every, c, ms))
        return rc;
    if (choice)
        for (int k = 0; k < 4; ++k)
            choice[k] = c[k];
    if (ms_out) {
        ms_out[0] = ms[0];
        ms_out[1] = ms[1];
    }
    return MDELAST_OK;
}

int mdelast_driver_set_launch(mdelast_driver *d, int32_t tpa_density, int32_t tpa_force,
                              int32_t blocks_density, int32_t blocks_force) {
    clear_error();
    if (!d)
        return fail(MDELAST_ERR_ARGUMENT, "null driver");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    if (int rc = d->set_launch(tpa_density, tpa_force, blocks_density, blocks_force))
        return rc;
    double md = 0., mf = 0.;
    return d->time_passes(1, 1, &md, &mf);
}

int mdelast_driver_list_capacity(mdelast_driver *d, int32_t *maxn, int32_t *regrowths) {
    clear_error();
    if (!d)
        return fail(MDELAST_ERR_ARGUMENT, "null driver");
    if (maxn)
        *maxn = d->A.maxn;
    if (regrowths)
        *regrowths = d->list_regrowths;
    return MDELAST_OK;
}

int mdelast_driver_set_force_staging(mdelast_driver *d, int32_t on) {
    clear_error();
    if (!d)
        return fail(MDELAST_ERR_ARGUMENT, "null driver");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    if (int rc = d->set_launch(d->tpa_d, d->tpa_f, d->target_d, d->target_f, on ? 1 : 0))
        return rc;
    double md = 0., mf = 0.;
    return d->time_passes(1, 1, &md, &mf);
}

int mdelast_driver_get_force_staging(mdelast_driver *d, int32_t *on, int32_t *available) {
    clear_error();
    if (!d)
        return fail(MDELAST_ERR_ARGUMENT, "null driver");
    if (on)
        *on = d->stage_f ? 1 : 0;
    if (available)
        *available = d->staging_available() ? 1 : 0;
    return MDELAST_OK;
}

int mdelast_driver_set_pair_list(mdelast_driver *d, double factor) {
    clear_error();
    if (!d)
        return fail(MDELAST_ERR_ARGUMENT, "null driver");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    return d->set_pair_list(factor);
}

int mdelast_driver_set_sample_ring(mdelast_driver *d, int32_t capacity) {
    clear_error();
    if (!d || capacity < 0)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    return d->alloc_ring(capacity);
}

int mdelast_driver_drain_samples(mdelast_driver *d, mdelast_sample *out, int64_t cap,
                                 int64_t *n_out, int64_t *n_lost) {
    return drain_samples_r(d, 0, out, cap, n_out, n_lost);
}

int mdelast_batch_drain_samples(mdelast_driver *d, int32_t replica, mdelast_sample *out,
                                int64_t cap, int64_t *n_out, int64_t *n_lost) {
    return drain_samples_r(d, replica, out, cap, n_out, n_lost);
}

int mdelast_driver_fluct_start(mdelast_driver *d) {
    clear_error();
    if (!d)
        return fail(MDELAST_ERR_ARGUMENT, "null driver");
    CK(cudaSetDevice(d->device));
    if (int rc = d->wait_step())
        return rc;
    k_samples_reset<<<(d->n_rep + 63) / 64, 64, 0, d->stream>>>(d->A, 2);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(d->stream));
    return MDELAST_OK;
}

int mdelast_driver_get_fluct(mdelast_driver *d, mdelast_fluct *out) {
    return get_fluct_r(d, 0, out);
}

int mdelast_batch_get_fluct(mdelast_driver *d, int32_t replica, mdelast_fluct *out) {
    return get_fluct_r(d, replica, out);
}

int mdelast_driver_get_observables(mdelast_driver *d, mdelast_observables *out) {
    return get_observables_r(d, 0, out);
}

int mdelast_driver_get_atoms(mdelast_driver *d, int32_t field, double *out) {
    return get_atoms_r(d, 0, field, out);
}

int mdelast_driver_get_chain(mdelast_driver *d, int32_t which, double *q, double *p_eta,
                             double *eta, int32_t *nchain) {
    return get_chain_r(d, 0, which, q, p_eta, eta, nchain);
}

int mdelast_driver_get_neighbors(mdelast_driver *d, int32_t *point, int32_t *neighbors,
                                 int64_t cap, int64_t *n_entries) {
    return get_neighbors_r(d, 0, point, neighbors, cap, n_entries);
}

int mdelast_batch_create(const mdelast_driver_config *cfgs, int32_t n_replicas,
                         mdelast_driver **out) {
    return create_system(cfgs, n_replicas, out);
}

int mdelast_batch_size(const mdelast_driver *d, int32_t *n_replicas, int64_t *n_atoms) {
    if (!d)
        return fail(MDELAST_ERR_ARGUMENT, "null driver");
    if (n_replicas)
        *n_replicas = d->n_rep;
    if (n_atoms)
        *n_atoms = d->N;
    return MDELAST_OK;
}

int mdelast_batch_get_observables(mdelast_driver *d, int32_t replica, mdelast_observables *out) {
    return get_observables_r(d, replica, out);
}

int mdelast_batch_get_status(mdelast_driver *d, uint32_t *status) {
    clear_error();
    if (!d || !status)
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    CK(cudaSetDevice(d->device));
    if (!d->obs_valid) {
        CK(cudaEventSynchronize(d->ev_step));
        d->obs_valid = true;
    }
    for (int r = 0; r < d->n_rep; ++r)
        status[r] = d->h_obs[r].status;
    return MDELAST_OK;
}

int mdelast_batch_get_atoms(mdelast_driver *d, int32_t replica, int32_t field, double *out) {
    return get_atoms_r(d, replica, field, out);
}

int mdelast_batch_get_chain(mdelast_driver *d, int32_t replica, int32_t which, double *q,
                            double *p_eta, double *eta, int32_t *nchain) {
    return get_chain_r(d, replica, which, q, p_eta, eta, nchain);
}

int mdelast_batch_get_neighbors(mdelast_driver *d, int32_t replica, int32_t *point,
                                int32_t *neighbors, int64_t cap, int64_t *n_entries) {
    return get_neighbors_r(d, replica, point, neighbors, cap, n_entries);
}

int mdelast_driver_pair_correlation(mdelast_driver *d, int32_t mode) {
    return pair_correlation_r(d, 0, mode);
}

int mdelast_driver_get_gr(mdelast_driver *d, double *gr, double *gr_partial) {
    return get_gr_r(d, 0, gr, gr_partial);
}

int mdelast_batch_pair_correlation(mdelast_driver *d, int32_t replica, int32_t mode) {
    return pair_correlation_r(d, replica, mode);
}

int mdelast_batch_get_gr(mdelast_driver *d, int32_t replica, double *gr, double *gr_partial) {
    return get_gr_r(d, replica, gr, gr_partial);
}

int mdelast_table_eval_device(const mdelast_pair *p, const mdelast_eam *e, int which,
                              const double *x, int64_t n, double *out) {
    clear_error();
    if (!x || !out || n < 0 || which < 0 || which > 2 || (which == 0 && !p) ||
        (which > 0 && !e))
        return fail(MDELAST_ERR_ARGUMENT, "bad argument");
    if (which == 0 && p->kind != PAIR_TABLE)
        return fail(MDELAST_ERR_UNSUPPORTED, "analytic pair potentials have no device table");
    if (!mdelast_device_available())
        return fail(MDELAST_ERR_NO_DEVICE, "no CUDA device");
    // a one-type table set holding just this function
    mdelast::QuinticTable const &tab = which == 0 ? p->table : (which == 1 ? e->rho : e->F);
    int const nint = tab.n;
    bool const bsp = tab.bspline != 0;
    size_t const kF = bsp ? 12 : 6;
    std::vector<double> const &src = bsp ? tab.cub : tab.coef;
    std::vector<double> rb, Ft;
    TablesView T{};
    T.interp = bsp ? MDELAST_BSPLINE : MDELAST_QUINTIC;
    if (which == 2) {
        Ft.assign(src.begin(), src.end());
        rb.assign(3 * kF, 0.);
        T.nfi = nint;
        T.inv_hf = tab.inv_h;
        T.inv_hf2 = tab.inv_h2;
        T.nri = 1;
    } else {
        rb.assign(static_cast<size_t>(nint) * 3 * kF, 0.);
        for (int k = 0; k < nint; ++k)
            std::memcpy(rb.data() + static_cast<size_t>(k) * 3 * kF + (which == 0 ? 0 : kF),
                        src.data() + kF * static_cast<size_t>(k), kF * sizeof(double));
        Ft.assign(kF, 0.);
        T.nri = nint;
        T.inv_hr = tab.inv_h;
        T.inv_hr2 = tab.inv_h2;
        T.nfi = 1;
    }
    T.npot = 1;
    T.ntypes = 1;
    T.pot_rcut[0] = which == 0 ? p->rcut : 0.;
    T.eam_rcut[0] = which == 1 ? e->rcut : 0.;
    double *d_rb = nullptr, *d_Ft = nullptr, *d_x = nullptr, *d_o = nullptr;
    int rc = MDELAST_OK;
    if ((rc = dalloc(&d_rb, rb.size())) || (rc = dalloc(&d_Ft, Ft.size())) ||
        (rc = dalloc(&d_x, static_cast<size_t>(n))) || (rc = dalloc(&d_o, 3 * static_cast<size_t>(n)))) {
        dfree(d_rb);
        dfree(d_Ft);
        dfree(d_x);
        dfree(d_o);
        return rc;
    }
    T.rb = d_rb;
    T.Ft = d_Ft;
    cudaError_t err = cudaMemcpy(d_rb, rb.data(), sizeof(double) * rb.size(), cudaMemcpyHostToDevice);
    if (!err)
        err = cudaMemcpy(d_Ft, Ft.data(), sizeof(double) * Ft.size(), cudaMemcpyHostToDevice);
    if (!err)
        err = cudaMemcpy(d_x, x, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (!err && n > 0) {
        k_table_eval<<<static_cast<unsigned>((n + 255) / 256), 256>>>(T, which, 0, d_x,
                                                                       static_cast<int>(n), d_o);
        err = cudaGetLastError();
    }
    if (!err)
        err = cudaMemcpy(out, d_o, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
    dfree(d_rb);
    dfree(d_Ft);
    dfree(d_x);
    dfree(d_o);
    if (err)
        return fail(MDELAST_ERR_CUDA, "device table evaluation: %s", cudaGetErrorString(err));
    return MDELAST_OK;
}

} // extern "C"
