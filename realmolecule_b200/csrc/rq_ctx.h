// rq_ctx.h -- the context object behind the C ABI (internal).
#pragma once
#include <string>
#include <vector>

#include "../../include/rq.h"
#include "rq_kernels.h"

struct rq_ctx;
int rq_fail(rq_ctx* c, int code, const std::string& msg);
int rq_cuda(rq_ctx* c, cudaError_t e, const char* where);

struct rq_mg_level {  // one level of the new flavour's multigrid hierarchy
  rq::Geo g;
  double h;
  void* P = nullptr;  // solution / correction (T)
  void* f = nullptr;  // right-hand side (T); the residual is never stored (fused into the restriction)
};

// Recording window of the new flavour's adjoint: the state each recorded step started from, so
// the reverse sweep can run back through the last `cap` steps (nm_adjoint.cu).
struct rq_adj {
  int cap = 0;                   // window length in steps (0: recording off)
  int np = 0;                    // P snapshot slots
  void* psi = nullptr;           // cap x S^3 (T): normalised psi each recorded step started from
  void* psum = nullptr;          // np x S^3 (T): P in effect (after each V-cycle; at the window start)
  double* scales = nullptr;      // cap x n_atoms: the per-domain scale of each normalising step
  struct Rec {
    int psi_slot, p_slot;
    bool vcycle, norm, label;    // V-cycle before the update, normalisation after it, label pass after it
  };
  std::vector<Rec> rec;          // recorded steps, oldest first (at most cap)
  long long next_psi = 0;        // ring positions
  int next_p = 0, cur_p = -1;
  // reverse-sweep buffers (allocated with the window)
  void* lam[2] = {nullptr, nullptr};  // adjoint of psi (T, S^3)
  void* muP[2] = {nullptr, nullptr};  // adjoint of the fine P (T, S^3; ping-pong through smoothing)
  void* muf = nullptr;                // adjoint of the fine right-hand side (T, S^3)
  double* gK = nullptr;               // dE/dK accumulated (S^3 doubles); dE/dv for the external potential
  struct Level { void* mu[2] = {nullptr, nullptr}; void* muf = nullptr; void* mur = nullptr; };
  std::vector<Level> lv;              // per multigrid level (level 0: only mur is used)
  double* dots = nullptr;             // per-domain <psi, lambda>
  double* coef = nullptr;             // per-domain (scale, beta) of a transposed normalisation
  double* wq = nullptr;               // per-domain (Z/N, Q/N) of the energy readout
};

// Tiled nuclear sums of the new flavour (nm_farfield.cu): tiles of <= 32^3 interior points,
// per tile the list of near nuclei and 16^3 Chebyshev node values / weights.
struct rq_ff {
  bool active = false;          // K and the gathers use the tiles for the current nuclei
  int nt = 0, base = 0, rem = 0, nTiles = 0;
  int nNuc = 0, capNuc = 0, capTiles = 0;
  double* nuc = nullptr;        // nNuc x (x, y, z, Z) bohr: the entries with Z_nuc > 0
  int* entry = nullptr;         // nNuc: their entry indices
  int* near_idx = nullptr;      // nTiles x nNuc: per tile the near nuclei, in order
  int* near_cnt = nullptr;      // nTiles
  double* nodes = nullptr;      // nTiles x 16^3: far-field node values (K) or node weights (gathers)
  double* tabs = nullptr;       // Chebyshev nodes and the Lagrange tables of every tile size
  double* Fraw = nullptr;       // nNuc x 3: the gathers' raw sums
};

struct rq_ctx {
  rq_config cfg{};
  rq_adj adj;
  rq_ff ff;
  rq::Geo g{};
  double h = 0, h2 = 0, h3 = 0, dv = 0, dt = 0, half_dv = 0, sigma = 0;
  int n_atoms = 0;
  std::vector<rq_atom> atoms;
  std::vector<rq_atom> atoms0;  // positions at creation (molecule.js groups nuclei by them)
  bool fp64 = false;
  cudaStream_t st = nullptr;
  cudaStream_t own_st = nullptr;
  int device = 0;

  // fields: psi, P double-buffered; labels double-buffered; T = float or double by precision
  void* U[2] = {nullptr, nullptr};
  void* P[2] = {nullptr, nullptr};
  void* K = nullptr;
  float* W = nullptr;
  float* bestU = nullptr;
  float* rho = nullptr;   // molecule.js rhoTotal / residual scratch (float)
  float* Pother = nullptr;  // molecule.js PotherBuf (stale P of the previous frame)
  float* resid = nullptr;   // molecule.js V-cycle residual
  int* lab[2] = {nullptr, nullptr};
  int cu = 0, cp = 0, cl = 0;

  // molecule.js coarse grid (2-level V-cycle) buffers
  rq::Geo gc{};
  float* Ec[2] = {nullptr, nullptr};
  float* fc = nullptr;

  // new flavour multigrid hierarchy (level 0 = fine)
  std::vector<rq_mg_level> mg;

  // atoms on the device
  float* atoms5 = nullptr;    // [i,j,k,Z,rc] f32 (cloud/solver.py:378-382)
  float* scratch_atoms5 = nullptr;  // per-call atom table for force variants
  float *sic = nullptr, *sic2 = nullptr;  // molecule.js flavour with SIC: self-potential ping-pong
  float* pdirect = nullptr;   // molecule.js direct path: persistent P_m of every domain (n_atoms x S^3)
  // molecule.js LOBPCG frames: HX, W, HW, P, HP (5 x S^3), the inner-product partial sums of
  // each workgroup (256 x 12) and the scalars (lambda, Ritz coefficients, the 12 sums of each pass)
  float* lob = nullptr;
  // molecule.js locked groups: per label the bit set of its groups (n_atoms, zero = none)
  unsigned long long* lock = nullptr;
  // molecule.js window.FREEZE_BOUNDARY: frames skip the level-set passes
  bool freeze = false;
  // molecule.js window.USER_INIT_POS: (i, j) per entry where init_has is set (the next initialisation)
  std::vector<double> init_pos;
  std::vector<int> init_has;
  // molecule.js shell splits per entry (n_atoms, zero = none)
  MjSplit* splits = nullptr;
  float* lob_part = nullptr;
  float* lob_scal = nullptr;
  // solver.py flavour: atom bins of the label step's argmax (rebuilt whenever atoms change)
  int bins_nb = 0, bins_bin = 0;
  int *bin_start = nullptr, *bin_idx = nullptr, *bin_far = nullptr;
  float* bin_zmax = nullptr;
  void* atoms_mj = nullptr;   // molecule.js records (u32 positions)
  double* atoms_nm = nullptr; // new flavour: x,y,z (bohr), Z_nuc per atom
  void* seeds = nullptr;      // new flavour: float4 (x, y, z, entry) per domain seed
  void* scale64 = nullptr;    // new flavour: per-domain scale (FP64 for both precisions)
  unsigned* rseed = nullptr;  // new flavour, fp32 fields: the step seed of the unbiased rounding (2 words by parity)
  double* K64 = nullptr;      // new flavour, fp32 fields: the FP64 nuclear (+ external) potential the readout uses
  unsigned char* nbm = nullptr;  // new flavour: same-label neighbour mask of the current labels (read by the update)
  void* Kext = nullptr;       // new flavour: external potential added to K (T), or null
  bool nm_pending = false;    // new flavour: psi awaits scale64 (applied by the next update or a flush)
  int sp_jdone = 0;           // solver.py flavour: the next Poisson step's first sweep is done (in P[1-cp])
  int nm_age = 0;             // new flavour: updates since psi was last normalised (0: normalised or pending)
  float* Zdom = nullptr;      // domain charge per label (f32)
  double* Zdom64 = nullptr;

  // FP64 per-domain sums and outputs
  double* dnorm = nullptr;    // n_atoms
  double* dpd = nullptr;      // n_atoms x 4
  double* dF = nullptr;       // n_atoms x 3
  double* dsum = nullptr;     // 8 global sums (energies / dipole)
  unsigned* unorm = nullptr;  // molecule.js fixed-point norms (n_atoms)
  float* scale = nullptr;     // n_atoms
  int* err = nullptr;         // device error word

  int steps_done = 0;
  int frame = 0;
  double cheb_omega = 1.0;  // molecule.js Chebyshev recurrence state (chebOmega, :1762)
  double cheb_E = 0.0;      // the page's E of the last frame (0 before the first, :1767)
  std::string last_error;

  // CUDA graphs of one schedule period, keyed by buffer parity (cu, cp, cl) and whether the
  // label updates of the period are active (label_until)
  cudaGraphExec_t graph[32] = {};
  int graph_post[32] = {};
  long long graph_launches[32] = {};

  // launch accounting and the optional per-kernel profile
  long long launches = 0;
  bool prof = false;
  struct ProfRec { cudaEvent_t a, b; int cls; double bytes; };
  std::vector<ProfRec> prec;
  std::vector<cudaEvent_t> evpool;
  size_t evused = 0;
};

// Launch wrapper: counts the launch and, while profiling, brackets it with CUDA events.
template <class F>
inline int rq_launch(rq_ctx* c, int cls, double bytes, F&& f) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (c->prof) {
    while (c->evpool.size() < c->evused + 2) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return rq_cuda(c, cudaGetLastError(), "cudaEventCreate");
      c->evpool.push_back(e);
    }
    a = c->evpool[c->evused++];
    b = c->evpool[c->evused++];
    cudaEventRecord(a, c->st);
  }
  cudaError_t e = f();
  if (c->prof) {
    cudaEventRecord(b, c->st);
    c->prec.push_back({a, b, cls, bytes});
  }
  c->launches++;
  return rq_cuda(c, e, "kernel launch");
}
#define LAUNCH(cls, bytes, call)                                               \
  do {                                                                         \
    int _lr = rq_launch(c, (cls), (double)(bytes), [&]() { return (call); });  \
    if (_lr != RQ_OK) return _lr;                                              \
  } while (0)

