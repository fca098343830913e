// Allocation-free energy entry point (included at the end of engine.cu, so it
// shares the engine's kernels and types; it adds no code to the other paths).
//
// Who needs it: a caller that must not allocate device memory while it runs --
// for example an NVQIR simulator plugin hosted inside another runtime whose
// device memory is owned by that runtime's pool, or a framework operator that
// works under a fixed memory budget -- cannot let the engine grow its
// workspaces with cudaMalloc on first use, as vqemps_energy_batch does. This
// entry point evaluates one parameter set with all of its intermediate data in
// one file-scope device array of fixed size, NOALLOC_SCRATCH_BYTES (22 MiB),
// which every GPU that loads the library holds until the process exits. The
// circuit and the Hamiltonian plan are still loaded beforehand with
// vqemps_set_circuit / vqemps_set_hamiltonian (which do allocate).
//
// Limits (checked before any launch, VQEMPS_INVALID otherwise): at most
// NOALLOC_MAX_SITES qubits, NOALLOC_MAX_SLOTS environments kept per trie level,
// NOALLOC_MAX_LEAVES distinct term endings. A 40-qubit, 5,000-term Pauli sum
// needs 2,067 slots and about 5,000 leaves.
//
// The scratch array is shared by every call in the process on a device and keeps
// the contents of the last call: calls whose execution overlaps on the GPU (on
// different streams, or from different threads) race on it and must be
// serialised by the caller. The first call on each device looks up the array's
// device address (cudaGetSymbolAddress with that device current); make that
// first call before any stream capture. The address is remembered together with
// the CUDA context it belongs to: after a device reset (or any other change of
// the context current on the device) the next call looks it up again, so it is
// that call, too, that must come before any stream capture. The call leaves the
// caller's current device as it found it.

#include <cuda.h>   // the CUcontext type only; the driver function is looked up at run time

#include <mutex>

namespace {

constexpr int NOALLOC_MAX_SITES = 64;
constexpr int NOALLOC_MAX_SLOTS = 2560;
constexpr int NOALLOC_MAX_LEAVES = 16384;

constexpr size_t na_align(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t NA_SITES = 0;
constexpr size_t NA_RIGHT = NA_SITES + na_align(sizeof(cplx) * NOALLOC_MAX_SITES * SITE_ELEMS);
constexpr size_t NA_ENV0 = NA_RIGHT + na_align(sizeof(cplx) * (NOALLOC_MAX_SITES + 1) * ENV_ELEMS);
constexpr size_t NA_ENV1 = NA_ENV0 + na_align(sizeof(cplx) * NOALLOC_MAX_SLOTS * ENV_ELEMS);
constexpr size_t NA_LEAF = NA_ENV1 + na_align(sizeof(cplx) * NOALLOC_MAX_SLOTS * ENV_ELEMS);
constexpr size_t NA_BONDS = NA_LEAF + na_align(sizeof(double) * NOALLOC_MAX_LEAVES);
constexpr size_t NA_STATUS = NA_BONDS + na_align(sizeof(int32_t) * (NOALLOC_MAX_SITES + 1));
constexpr size_t NOALLOC_SCRATCH_BYTES = 22u << 20;
static_assert(NA_STATUS + 256 <= NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the array");

// The scratch memory itself. Host code must not use this name as an address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mutex;
struct NoallocAddr {
  CUcontext context;
  unsigned char *addr;
};
NoallocAddr g_noalloc_addr[128] = {};

// The CUDA context current on the calling thread (null if the driver cannot be
// asked). cuCtxGetCurrent is fetched through the runtime, so the library does
// not link against the driver library and still loads on machines without one.
CUcontext noalloc_current_context() {
  typedef CUresult (*GetCurrent)(CUcontext *);
  static GetCurrent fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (GetCurrent) nullptr;
    return reinterpret_cast<GetCurrent>(p);
  }();
  CUcontext c = nullptr;
  if (fn == nullptr || fn(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

// Device address of the scratch array on `device` (which must be current), looked
// up again whenever the current context is not the one of the remembered address.
int noalloc_scratch(vqemps_ctx *ctx, unsigned char **out) {
  if (ctx->device < 0 || ctx->device >= 128) return fail(ctx, VQEMPS_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoallocAddr &slot = g_noalloc_addr[ctx->device];
  const CUcontext current = noalloc_current_context();
  if (slot.addr == nullptr || current == nullptr || slot.context != current) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(ctx, VQEMPS_CUDA_ERROR, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    slot.addr = static_cast<unsigned char *>(ptr);
    slot.context = current;
  }
  *out = slot.addr;
  return VQEMPS_OK;
}

// Makes `device` current for one call and gives the caller's device back after.
struct NoallocDeviceScope {
  int previous = -1;
  cudaError_t status = cudaSuccess;
  explicit NoallocDeviceScope(int device) {
    if (cudaGetDevice(&previous) != cudaSuccess) previous = -1;
    if (previous != device) status = cudaSetDevice(device);
  }
  ~NoallocDeviceScope() {
    int now = -1;
    if (previous >= 0 && cudaGetDevice(&now) == cudaSuccess && now != previous) cudaSetDevice(previous);
  }
};

}  // namespace

extern "C" int vqemps_energy_noalloc(vqemps_ctx *ctx, int handle, const double *theta_dev,
                                     double *energy_dev, double *per_term_dev, int32_t *status_dev,
                                     void *stream) {
  if (!ctx) return VQEMPS_INVALID;
  if (!ctx->have_circuit) return fail(ctx, VQEMPS_INVALID, "no circuit");
  Hamiltonian *h = find_ham(ctx, handle);
  if (!h) return fail(ctx, VQEMPS_INVALID, "unknown Hamiltonian handle");
  if ((!theta_dev && ctx->P > 0) || !energy_dev) return fail(ctx, VQEMPS_INVALID, "bad arguments");
  const int n = ctx->n;
  if (n > NOALLOC_MAX_SITES)
    return fail(ctx, VQEMPS_INVALID, "vqemps_energy_noalloc: " + std::to_string(n) + " qubits exceed the limit of " +
                                         std::to_string(NOALLOC_MAX_SITES));
  if (h->max_slot > NOALLOC_MAX_SLOTS)
    return fail(ctx, VQEMPS_INVALID, "vqemps_energy_noalloc: the Pauli sum keeps " + std::to_string(h->max_slot) +
                                         " environments on one site, above the limit of " +
                                         std::to_string(NOALLOC_MAX_SLOTS));
  if (h->nleaf > NOALLOC_MAX_LEAVES)
    return fail(ctx, VQEMPS_INVALID, "vqemps_energy_noalloc: " + std::to_string(h->nleaf) +
                                         " distinct term endings exceed the limit of " +
                                         std::to_string(NOALLOC_MAX_LEAVES));
  NoallocDeviceScope device_scope(ctx->device);
  CUDA_TRY(ctx, device_scope.status);
  unsigned char *base = nullptr;
  int rc = noalloc_scratch(ctx, &base);
  if (rc) return rc;
  cplx *sites = reinterpret_cast<cplx *>(base + NA_SITES);
  cplx *right = reinterpret_cast<cplx *>(base + NA_RIGHT);
  cplx *envs[2] = {reinterpret_cast<cplx *>(base + NA_ENV0), reinterpret_cast<cplx *>(base + NA_ENV1)};
  double *leafval = reinterpret_cast<double *>(base + NA_LEAF);
  int32_t *bonds = reinterpret_cast<int32_t *>(base + NA_BONDS);
  int32_t *status = reinterpret_cast<int32_t *>(base + NA_STATUS);
  cudaStream_t st = as_stream(stream);
  const int nleaf = std::max(h->nleaf, 1);
  // Every value read below is written earlier in this call; the leaf values
  // are cleared anyway so a stale result of a previous call can never leak.
  CUDA_TRY(ctx, cudaMemsetAsync(leafval, 0, sizeof(double) * nleaf, st));

  EvolveParams ep{};
  ep.gates = ctx->d_gates;
  ep.ngates = (int)ctx->gates.size();
  ep.mats = ctx->d_mats;
  ep.n = n;
  ep.P = ctx->P;
  ep.theta = theta_dev;
  ep.sites = sites;
  ep.bonds = bonds;
  ep.status = status;
  ep.init0 = ctx->init0;
  ep.init1 = ctx->init1;
  ep.max_bond = ctx->max_bond;
  ep.abs_cut = ctx->abs_cut;
  ep.rel_cut = ctx->rel_cut;
  evolve_kernel<<<1, EVOLVE_THREADS, EvolveSmem::bytes(n), st>>>(ep);
  CUDA_TRY(ctx, cudaGetLastError());
  right_env_kernel<<<1, RIGHT_THREADS, 0, st>>>(sites, n, right, nullptr, status, leafval, nleaf,
                                               h->identity_leaf);
  CUDA_TRY(ctx, cudaGetLastError());
  for (int s = 0; s < n; ++s) {
    const int ng = h->group_off[s + 1] - h->group_off[s];
    if (ng == 0) break;
    LevelParams lp{};
    lp.sites = sites;
    lp.right = right;
    lp.env_prev = envs[(s + 1) & 1];
    lp.env_cur = envs[s & 1];
    lp.groups = h->d_groups + h->group_off[s];
    lp.nodes = h->d_nodes + h->node_off[s];
    lp.leafval = leafval;
    lp.ngroups = ng;
    lp.nslot_prev = s > 0 ? std::max(h->nslot[s - 1], 1) : 1;
    lp.nslot_cur = std::max(h->nslot[s], 1);
    lp.nleaf_total = nleaf;
    lp.n = n;
    lp.s = s;
    level_kernel<<<dim3((ng + LEVEL_WARPS - 1) / LEVEL_WARPS, 1), LEVEL_WARPS * 32, sizeof(LevelSmem), st>>>(lp);
    CUDA_TRY(ctx, cudaGetLastError());
  }
  reduce_kernel<<<1, REDUCE_THREADS, 0, st>>>(leafval, h->d_leaf_coef, h->nleaf, h->d_term_leaf, h->T, status,
                                             energy_dev, per_term_dev);
  CUDA_TRY(ctx, cudaGetLastError());
  if (status_dev)
    CUDA_TRY(ctx, cudaMemcpyAsync(status_dev, status, sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
  return VQEMPS_OK;
}
