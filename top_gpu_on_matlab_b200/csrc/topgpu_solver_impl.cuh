// topgpu_solver_impl.cuh -- internal state of the fused solver, shared by
// topgpu_solver.cu (operators, V-cycle, PCG, assembly) and topgpu_opt.cu
// (filters, sensitivities, OC loop).
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <cstdlib>
#include <vector>
#include <utility>
#include "topgpu_grid.cuh"
#include "topgpu_walsh.cuh"
#include "topgpu_tc.cuh"

namespace topgpu {

// ---------------------------------------------------------------------------
struct DevLevel {
    int ny = 0, nx = 0, nz = 0, span = 0;
    Geom g{};
    int64_t Ne = 0, Nn = 0, ng = 0;
    uint8_t *flags = nullptr;
    int32_t *nodeGrid = nullptr, *eleGrid = nullptr, *upMap = nullptr;
    double *KsC = nullptr, *KsP64 = nullptr; float *KsP32 = nullptr;
    double *W64 = nullptr; float *W32 = nullptr;   // element outputs of the two-pass coarse product
    double *diag = nullptr, *invD64 = nullptr; float *invD32 = nullptr;
    double *r64 = nullptr, *x64 = nullptr, *t64 = nullptr;
    float *r32 = nullptr, *x32 = nullptr, *t32 = nullptr;
    uint8_t *tileFixed = nullptr;
};

}  // namespace topgpu

struct top_solver {
    using DevLevel = topgpu::DevLevel;
    using PcgState = topgpu::PcgState;
    using Reduce = topgpu::Reduce;
    top_solver_params p{};
    cudaStream_t st = nullptr;
    // CUDA graph of a chunk of PCG iterations (captured on an internal stream,
    // re-captured when an operand pointer or the operator configuration changes)
    struct PcgGraph {
        cudaGraphExec_t exec = nullptr;
        const double *b = nullptr; double *x = nullptr; int gen = -1, chunk = 0, nrhs = 1; int64_t nodes = 0;
    };
    std::vector<PcgGraph> graphs;    // one per (right-hand side, solution) pair in use
    cudaStream_t capStream = nullptr; cudaEvent_t capIn = nullptr, capOut = nullptr;
    bool useGraphs = true;
    bool coarseLanes = std::getenv("TOPGPU_COARSE_LANES") != nullptr;   // 8-lanes-per-node coarse kernel
    int coarsePersistent = 0;        // levels from 1 (1) or from 2 (2) down of the V-cycle in one cooperative launch; 0 off
    // coarse levels with at least this many packed tiles take the two-pass
    // product (element outputs, then node sums; identical results)
    int coarseTwoPassMin = std::getenv("TOPGPU_COARSE_TWOPASS_MIN") ? std::atoi(std::getenv("TOPGPU_COARSE_TWOPASS_MIN")) : 0;
    bool pdl = std::getenv("TOPGPU_NO_PDL") == nullptr;
    // span-4 transfers read and write four fine y slots as one aligned vector
    // (identical results; TOPGPU_NO_VEC4 selects the per-slot kernels)
    bool vec4 = std::getenv("TOPGPU_NO_VEC4") == nullptr;   // programmatic dependent launch on the PCG path
    bool inCapture = false;          // launches are being captured into a graph (no dependent launch there)
    // PCG direction update: false = the reference's beta = rho / rhoOld (TOP_GPU.m:650-653);
    // true = flexible (Polak-Ribiere) beta = z.(r - r_old) / rhoOld = -z.(A p_old) / (p_old.A p_old)
    bool flexible = false;
    int opGen = 0;                   // bumped whenever captured launches would change
    int nL = 0, nLoads = 0;
    std::vector<DevLevel> L;
    std::vector<void *> allocs;      // raw allocations (freed on destroy)
    topgpu::KeParam<double> Ke64{}; topgpu::KeParam<float> Ke32{};
    // level-0 product: kind 0 = node-centric dense Ke, 1 = Walsh-basis tiles
    // of ty x tx element columns (one per thread), 2 = the same with two
    // element columns per thread (ty x tx threads), 3 = Walsh with direct
    // loads, 4 = paired direct loads, 5 = tensor cores (FP32, 16 x 8), 6 =
    // paired with TMA-staged node layers (FP32; tiles of 2 ty x tx), on
    // ctas CTAs (0: as many as fit at once); per precision, set by
    // top_solver_set_l0_kernel or the autotuner
    struct L0Kernel { int kind = 0, ty = 16, tx = 16, ctas = 0; uint8_t *mask = nullptr; };
    int numSMs = 148;
    L0Kernel l0k[2];                 // [0] FP64, [1] FP32
    L0Kernel l0kFallback;            // kind 6 with a converting operand: the direct-load kind, 16 x 8
    bool stageErr = false;           // kind 6: a tensor map could not be encoded
    bool walshOK = false;            // Ke has the cube's reflection symmetry
    topgpu::TcOperandB *tcB = nullptr;   // kind 5: Ke as TF32 hi/lo tensor-core operand (device)
    int *tcErr = nullptr;            // kind 5: set by a kernel whose MMA wait gave up
    int *opErr = nullptr;            // set by a two-pass coarse product whose tile copy wait gave up
    // The V-cycle from level tailL down as one operator M (dense, symmetric, on
    // that level's active DOFs), formed at assembly and applied by one GEMV.
    // tailL 0: no level qualifies.  tailMode: -1 the default (on in mixed
    // precision, off in FP64), 0 off, 1 on.
    static constexpr int64_t kTailMaxDofs = 2500;
    int tailL = 0, tailMode = -1;
    bool tailReady = false;          // tailMp matches the current assembly
    std::vector<double *> tailPt;    // prolongation of level l+1 into l, transposed: [j + m k], l = tailL..nL-2
    std::vector<int32_t *> tailNbr;  // per compact node of those levels: 27 neighbour nodes (-1: none)
    std::vector<int32_t *> tailNodeCompact, tailEleCompact;   // grid slot -> compact node / element
    std::vector<double *> tailMs;    // M of levels tailL..nL-2, column-major, FP64
    double *tailK = nullptr, *tailQ = nullptr, *tailT = nullptr, *tailJ = nullptr;
    void *tailMp = nullptr;          // M of level tailL by rows at stride tailLd, in the V-cycle's precision
    void *tailR = nullptr;           // its operand in compact order (stride tailLd per right-hand side, zero beyond n)
    int64_t tailLd = 0;
    // test of that give-up path: the next two-pass product withholds one tile copy
    // (one-shot, armed by top_solver_test_withhold_tile)
    bool withholdTile = false;
    topgpu::WalshParam<double> W64{}; topgpu::WalshParam<float> W32{};
    topgpu::WalshPairParam<double> WP64{}; topgpu::WalshPairParam<float> WP32{};
    double *KeDev = nullptr, *P4 = nullptr, *P2 = nullptr;
    double *Ec = nullptr, *Eg64 = nullptr; float *Eg32 = nullptr;
    int32_t *mapUnique = nullptr; double *uFree = nullptr, *uFixed = nullptr; int64_t nU = 0;
    double *Qs = nullptr; int32_t *eye = nullptr;
    int32_t *bndList = nullptr; int64_t nBnd = 0;   // level-1 cells with fixed-DOF children
    double *x = nullptr, *r = nullptr, *z = nullptr, *pv = nullptr, *v = nullptr, *tmp = nullptr;
    float *z32 = nullptr;            // FP32 preconditioned residual of the mixed path
    double *rscr64 = nullptr; float *rscr32 = nullptr;   // separable restriction scratch
    double *b = nullptr;             // [nLoads][3 x cs]
    double *weights = nullptr;
    PcgState *state = nullptr, *hstate = nullptr;
    double *partials = nullptr; unsigned *counter = nullptr; int64_t nPartials = 0;
    double *scal = nullptr;          // device scalars for standalone reductions
    int *zeroDone = nullptr;
    int64_t nC = 0; double *Ac = nullptr, *Ainv = nullptr, *Wc = nullptr, *cr = nullptr;
    double *Dc = nullptr;            // inverses of the coarsest factor's 32 x 32 diagonal blocks
    int32_t *eleCompactC = nullptr, *nodeCompactC = nullptr;
    bool assembled = false;
    // super-element mode (TOP_GPU.m:1101-1104, 721-741): level-0 elements are
    // 4x4x4 sub-voxel blocks with per-element K_mat = I_mat * E_sub
    bool super = false;
    double *Esub = nullptr;          // [64 x Ne] sub-voxel moduli
    double *Imat = nullptr;          // [576 x 64]
    double *stage = nullptr;         // host-upload staging for [64 x Ne] vectors
    int nely = 0, nelx = 0, nelz = 0;   // the model's voxel (super-element) counts
    int64_t launches = 0;            // kernels launched by this solver (all entry points)
    void *filterState = nullptr, *optState = nullptr, *adjState = nullptr;   // topgpu_opt.cu
    std::vector<double> Fhost; int64_t nd0 = 0;

    template <typename T> T *dalloc(size_t n)
    {
        void *ptr = nullptr;
        if (cudaMalloc(&ptr, sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
        cudaMemset(ptr, 0, sizeof(T) * (n ? n : 1));
        allocs.push_back(ptr);
        return static_cast<T *>(ptr);
    }
    // grid array with margins: ncomp components of stride cs
    template <typename T> T *galloc(int64_t cs, int ncomp)
    {
        T *b = dalloc<T>((size_t)cs * ncomp);
        return b ? b + topgpu::kMargin : nullptr;
    }
    // packed coarse matrices in the tile-interleaved layout (topgpu_grid.cuh)
    template <typename T> T *ksalloc(int64_t cs)
    {
        T *b = dalloc<T>((size_t)topgpu::ks_alloc_vals(cs));
        return b ? b + topgpu::kKsFront : nullptr;
    }
    // element outputs of the two-pass coarse product, nv right-hand sides
    // (stride w_alloc_vals(cs)), each behind a zero guard tile
    template <typename T> T *walloc(int64_t cs, int nv)
    {
        T *b = dalloc<T>((size_t)topgpu::w_alloc_vals(cs) * nv);
        return b ? b + topgpu::kWFront : nullptr;
    }
    Reduce red(double *result) const { return Reduce{partials, counter, result}; }
    // per-right-hand-side sums into consecutive PcgState's (batched launches)
    Reduce redk(double *result) const { return Reduce{partials, counter, result, nPartials, topgpu::kStateDoubles}; }
    int kMax = 1;                    // right-hand sides the buffers hold (load cases)
};

namespace topgpu {
// named host range for profilers (NVTX; nothing happens without one attached)
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};
// launch on the PCG path: with s->pdl, outside graph capture, the kernel may
// be scheduled while its predecessor in the stream finishes (it must begin
// with pdl_enter()); captured graphs keep plain dependencies (measured: the
// dependent launch gains nothing inside them)
template <typename... KArgs, typename... Args>
inline void launch_k(const top_solver *s, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                     Args &&...args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid; cfg.blockDim = block; cfg.dynamicSmemBytes = smem; cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = (s->pdl && !s->inCapture) ? 1 : 0;
    cfg.attrs = at; cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}
}  // namespace topgpu

// every kernel launch of the solver is counted on the solver it serves
#define TOPGPU_COUNT_LAUNCH() (++s->launches)

namespace topgpu {
// y-epilogue applied to (K_0 in)(node) for every level-0 node, with the
// level-0 kernel configured for precision T (topgpu_l0.cu)
template <typename T, class In, class Out>
void l0_op(top_solver *s, const In &in, const Out &out, Reduce red, const int *done, int nv = 1);
// configure the level-0 kernel of precision slot p (0 FP64, 1 FP32)
int set_l0_kernel(top_solver *s, int p, int kind, int ty, int tx, int ctas);
// time every level-0 kernel configuration, keep the fastest per precision
int autotune_l0(top_solver *s, int nrep, int64_t flushBytes, double *msBest, int *configs);
// PCG (TOP_GPU.m:602-667) on level-0 grid vectors: b and x in the solver's
// SoA grid layout, x holds the warm start when warm != 0 and the solution.
int pcg_grid(top_solver *s, const double *bGrid, double *xGrid, int warm, int *itsOut, double *resOut);
// the same on nrhs right-hand sides at once (vectors at stride 3 CS)
int pcg_block(top_solver *s, const double *bGrid, double *xGrid, int nrhs, int warm, int *itsOut, double *resOut);
void free_opt_state(top_solver *s);
// element moduli from a compact element vector (SIMP when simp != 0)
int set_modulus_dev(top_solver *s, const double *src, int where, int simp);
template <typename TI, typename TO>
__global__ void compact_to_grid_kernel(const TI *__restrict__ v, TO *__restrict__ g,
                                       const int32_t *__restrict__ nodeGrid, int64_t Nn, int64_t cs);
template <typename TI, typename TO>
__global__ void grid_to_compact_kernel(const TI *__restrict__ g, TO *__restrict__ v,
                                       const int32_t *__restrict__ nodeGrid, int64_t Nn, int64_t cs);
inline int nb256(int64_t n) { return (int)((n + 255) / 256 < (1 << 20) ? (n + 255) / 256 : (1 << 20)); }
}  // namespace topgpu
