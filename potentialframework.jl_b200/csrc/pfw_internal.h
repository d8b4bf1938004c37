// pfw_internal.h — workspace state and internal interfaces of libpfw_b200.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pfw_b200.h"
#include "pfw_common.cuh"

namespace pfw {

struct Error : std::runtime_error {
  pfw_status code;
  Error(pfw_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define PFW_CUDA(call)                                                                             \
  do {                                                                                             \
    cudaError_t _e = (call);                                                                       \
    if (_e != cudaSuccess)                                                                         \
      throw ::pfw::Error(PFW_ECUDA, std::string(#call) + ": " + cudaGetErrorString(_e));           \
  } while (0)

// Bumped by every device reallocation in the process: a captured CUDA graph
// recorded at an older epoch may hold freed pointers and is re-captured.
inline std::atomic<uint64_t> g_alloc_epoch{0};

// Growable device buffer (never shrinks; contents not preserved on growth).
struct DevBuf {
  void* ptr = nullptr;
  size_t cap = 0;
  void* ensure(size_t bytes) {
    if (bytes > cap) {
      g_alloc_epoch.fetch_add(1);
      if (ptr) cudaFree(ptr);
      ptr = nullptr;
      size_t want = bytes < 256 ? 256 : bytes + bytes / 4;
      PFW_CUDA(cudaMalloc(&ptr, want));
      cap = want;
    }
    return ptr;
  }
  template <class T>
  T* as() const { return static_cast<T*>(ptr); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
  }
};

// Host description of one system before device preparation.
struct HostSystem {
  double H[9];
  uint8_t pbc[3];
  int32_t atom_begin, natoms;
};

// Device geometry after prepare (sorted atoms in cells).
struct Prepared {
  double cutoff = -1;
  int32_t n = 0;
  int32_t ncells = 0;
  int32_t nsys = 0;
  int32_t max_cell = 0;  // largest cell population
  int32_t species_limit = INT32_MAX;  // species limit the sorted positions were validated against
  bool any_image = false;
  std::vector<SysGeom> sys;  // host copy
  bool valid = false;
};

struct PairModel {
  int kind = -1;  // 0 smooth, 1 LJ
  int nz = 0;
  std::vector<double> A;
  double eps = 0, sigma = 0, cutoff = 0;
};

struct AceDevice;  // ace.cu
struct SurDevice;  // ace.cu (surrogate)
struct SkinState;  // skin.cu
struct PairGraph;  // pair.cu
struct MlpScratch;  // mlp.cu

}  // namespace pfw

struct pfw_ws {
  pfw_options opt{};
  cudaStream_t stream = nullptr;
  std::string err;
  // geometry input (original order)
  int32_t n = 0;
  int32_t max_species = 0;  // largest species channel of a host-uploaded batch (single systems: checked on the device)
  // channel count of the model the next cell-list build serves: k_gather
  // flags channels outside [0, species_limit) on the device (device uploads)
  int32_t species_limit = INT32_MAX;
  // pfw_evaluate reads the cell-list flags with its outputs (one synchronisation):
  // prepare_check only queues their copy into flags_host while defer_check is set
  bool defer_check = false, check_pending = false;
  int32_t* flags_host = nullptr;  // pinned, 8 words
  std::vector<pfw::HostSystem> systems;
  uint64_t geometry_version = 0;  // bumped when the systems (count, sizes, cells) change
  int32_t n_owned = -1;           // atoms [0, n_owned) own E/W (domain decomposition); -1: all
  double skin = 0.0;              // pair neighbour-list skin (Å); 0: rebuild every call
  pfw::SkinState* skin_state = nullptr;
  pfw::PairGraph* pair_graph = nullptr;  // captured single-system pair evaluation
  pfw::MlpScratch* mlp_scratch = nullptr;  // device scratch of the MLP training steps
  uint64_t model_version = 0;            // bumped by every pair-model change
  pfw::DevBuf X, species, atom_sys;  // X: 3n doubles
  // prepared geometry
  pfw::Prepared prep;
  pfw::DevBuf sysgeom, wrapped, bincoord, wind, cellid, slot, cell_count, cell_start, cell_sys, tmp_idx,
      perm, inverse, pos, pos32, scan_tmp, minmax;
  // pair evaluation
  pfw::PairModel pair;
  pfw::DevBuf cellpart, out_E, out_F, out_W, out_feat, counters, red_partial, out_design, out_base;
  pfw::DevBuf slab_scratch;  // band flags and offsets of pfw_slab_bands
  pfw::DevBuf pair_slots;  // per-(slot, sorted atom) partial forces of the half-stencil pair kernel
  int64_t last_pairs = -1;
  // neighbour snapshot
  pfw::DevBuf nb_count, nb_offsets, nb_j, nb_S, nb_R;
  int64_t nb_total = -1;
  // ACE
  pfw::AceDevice* ace = nullptr;
  pfw::SurDevice* sur = nullptr;
  int32_t last_model = -1;  // model selector of the last evaluation
  // bookkeeping
  uint64_t launches = 0;
  cudaStream_t own_stream = nullptr;  // the workspace's stream (stream may be the caller's)
  // stage diagnostics: event pairs per stage
  bool diag = false;
  cudaEvent_t ev[8] = {};
  bool ev_used[4] = {};
  void stage_begin(int s) {
    if (diag) {
      cudaEventRecord(ev[2 * s], stream);
      ev_used[s] = true;
    }
  }
  void stage_end(int s) {
    if (diag) cudaEventRecord(ev[2 * s + 1], stream);
  }
};

namespace pfw {
// geometry.cu
void prepare(pfw_ws* ws, double cutoff);
bool prepare_plan(pfw_ws* ws, double cutoff);  // host plan; true if it already wrapped (open axes)
void prepare_launch(pfw_ws* ws, bool wrap);    // device-only build, capturable
void prepare_check(pfw_ws* ws);                // synchronise, raise on device flags (or queue them, deferred)
void prepare_check_finish(pfw_ws* ws);         // after the caller's synchronisation: raise on deferred flags
void exclusive_scan_i32(pfw_ws* ws, const int32_t* in, int32_t* out, int64_t n);  // out has n+1 entries
void exclusive_scan_i64(pfw_ws* ws, const int32_t* in, int64_t* out, int64_t n);
// reduce.cu: deterministic partial sums → E[0] and W[9] (either may be null)
void reduce_pair_parts(pfw_ws* ws, const double* parts, int nparts, int stride, double* E, double* W);
void reduce_site_parts(pfw_ws* ws, const double* parts, int nparts, double* E, double* W);
// skin.cu: pair evaluation from a cached c+skin list while no atom moved more
// than skin/2 since it was built (returns false when the list path does not apply)
bool skin_pair_evaluate(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev);
void skin_free(pfw_ws* ws);
void skin_stats(pfw_ws* ws, int64_t* builds, int64_t* reuses);
// pair.cu
// per_system: E[s] and W[9s..] for every system of a batch
void pair_evaluate(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev, bool per_system = false);
void pair_graph_free(pfw_ws* ws);
// pair_half.cu: every unordered pair once (3×3×3 stencils with per-cell shifts)
struct PairParams;
bool pair_half_eligible(const Prepared& P);
void pair_half_setup();
void pair_half_kernel(pfw_ws* ws, const PairParams& prm, double* parts, unsigned long long* np);
void pair_half_fold(pfw_ws* ws, double* F);
void slab_bands(pfw_ws* ws, int64_t n, const double* X, const int32_t* species, const double fr[3], double lo,
                double hi, double d, const double sl[3], const double su[3], double* lower, double* upper,
                int32_t* counts);
// snapshot.cu
int64_t neighbour_build(pfw_ws* ws, double cutoff, bool with_R = true);
void neighbour_fill(pfw_ws* ws, int64_t* offsets, int32_t* j, int32_t* S, double* R);
// ace.cu
void ace_load(pfw_ws* ws, const pfw_ace_tables* t);
void ace_set_schedule(pfw_ws* ws, int chunk, int groups);
void ace_free(pfw_ws* ws);
void ace_evaluate(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev);
void ace_site_energies(pfw_ws* ws, double* host);
// zero the E/W partials of sites whose atom is a ghost copy (perm[s] >= n_owned)
void mask_unowned_sites(pfw_ws* ws, double* site_out, int n);
int ace_feature_count(pfw_ws* ws);
void ace_design_shape(pfw_ws* ws, int64_t* rows, int64_t* cols);
void ace_design_matrix(pfw_ws* ws, double* A_dev, int64_t ld, int64_t rows_capacity, double* base_dev);
void ace_evaluate_batch(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev, double* feat_dev);
void ace_batch_graph(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev, double* feat_dev);
void ace_batch_graph_sync(pfw_ws* ws);
double probe_fp64(pfw_ws* ws);
// ace.cu: surrogate
void sur_load(pfw_ws* ws, const pfw_ace_tables* features, const pfw_mlp_params* mlp);
void sur_free(pfw_ws* ws);
void sur_features(pfw_ws* ws, double* out_dev);
void sur_evaluate(pfw_ws* ws, uint32_t req, double* E_dev, double* F_dev, double* W_dev);
void sur_stats(pfw_ws* ws, int64_t* fallback, int64_t* sites);
void sur_site_energies(pfw_ws* ws, double* host);
int sur_feature_width(pfw_ws* ws);
// mlp.cu: ensemble training (mean-squared site-energy loss, Adam)
void mlp_param_grad(pfw_ws* ws, const pfw_mlp_shape* shape, const float* params, int64_t n, const float* X,
                    const float* y, const int32_t* species, double* loss, float* grad);
void mlp_train(pfw_ws* ws, const pfw_mlp_shape* shape, float* params, int64_t n, const float* X, const float* y,
               const int32_t* species, const pfw_mlp_train_options* opt, float* epoch_loss);
// mlp.cu: energy + force training steps on device buffers
void mlp_ef_step(pfw_ws* ws, const pfw_mlp_shape* shape, float* params_dev, float* m1_dev, float* m2_dev, int64_t n,
                 const float* X_dev, const float* y_dev, const int32_t* species, const float* V_dev,
                 const float* c_dev, float wE, float lr, int64_t step, float* grad_dev, double* loss);
void mlp_input_grad(pfw_ws* ws, const pfw_mlp_shape* shape, const float* params_dev, int64_t n, const float* X_dev,
                    const int32_t* species, float* G_dev);
void mlp_scratch_free(pfw_ws* ws);
// ace.cu: forces of a per-site dE/dfeature field through the feature model
void sur_pullback(pfw_ws* ws, const double* dEdx_dev, double* F_dev);

inline int grid_for(int64_t n, int block) { return (int)((n + block - 1) / block); }

// A model with nz species channels is about to be evaluated: host-uploaded
// species are checked here; device-uploaded ones by the next cell-list build.
inline void check_species(pfw_ws* ws, int nz, const char* msg) {
  if (ws->max_species >= nz) throw Error(PFW_EINVAL, msg);
  ws->species_limit = nz;
}
}  // namespace pfw
