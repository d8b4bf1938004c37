// capi.cu — the extern "C" boundary of libpfw_b200.so (include/pfw_b200.h).
//
// Every entry point catches internal errors and returns a pfw_status with
// the message kept in the workspace (pfw_last_error).  Nothing here falls
// back to a CPU computation: a missing device is an error.
#include <algorithm>
#include <cmath>
#include <vector>
#include <cstdio>
#include <new>

#include "pfw_internal.h"

using pfw::Error;

namespace {

pfw_status fail(pfw_ws* ws, pfw_status code, const std::string& msg) {
  if (ws) ws->err = msg;
  return code;
}

template <class F>
pfw_status guarded(pfw_ws* ws, F&& f) {
  if (!ws) return PFW_EINVAL;
  try {
    PFW_CUDA(cudaSetDevice(ws->opt.device));
    ws->err.clear();
    f();
    return PFW_OK;
  } catch (const Error& e) {
    return fail(ws, e.code, e.what());
  } catch (const std::bad_alloc&) {
    return fail(ws, PFW_ECUDA, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(ws, PFW_EINVAL, e.what());
  }
}

void upload_geometry(pfw_ws* ws, int64_t n, const double* X, const double* H, const uint8_t pbc[3],
                     const int32_t* species, bool device_ptrs) {
  if (n < 0 || n > (int64_t)INT32_MAX / 4) throw Error(PFW_EINVAL, "atom count out of range");
  if (n > 0 && (!X || !species)) throw Error(PFW_EINVAL, "positions and species are required");
  if (!H || !pbc) throw Error(PFW_EINVAL, "cell and pbc are required");
  pfw::HostSystem hs;
  for (int k = 0; k < 9; ++k) hs.H[k] = H[k];
  for (int a = 0; a < 3; ++a) hs.pbc[a] = pbc[a] ? 1 : 0;
  hs.atom_begin = 0;
  hs.natoms = (int32_t)n;
  ws->systems.assign(1, hs);
  ws->n = (int32_t)n;
  ws->n_owned = -1;
  ws->geometry_version += 1;
  cudaMemcpyKind kind = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  ws->X.ensure(sizeof(double) * 3 * std::max<int64_t>(n, 1));
  ws->species.ensure(sizeof(int32_t) * std::max<int64_t>(n, 1));
  if (n > 0) {
    PFW_CUDA(cudaMemcpyAsync(ws->X.ptr, X, sizeof(double) * 3 * n, kind, ws->stream));
    PFW_CUDA(cudaMemcpyAsync(ws->species.ptr, species, sizeof(int32_t) * n, kind, ws->stream));
  }
  // species channels are validated on the device while the cell list is
  // sorted (outside [0, the model's channel count) raises PFW_EINVAL at the
  // end of the call), for host and device uploads alike
  ws->max_species = 0;
  ws->prep.valid = false;
  ws->nb_total = -1;
  ws->last_pairs = -1;
}

void upload_batch(pfw_ws* ws, int32_t nsys, const int64_t* offsets, const double* X, const double* H,
                  const uint8_t* pbc, const int32_t* species, bool device_ptrs) {
  if (nsys < 1) throw Error(PFW_EINVAL, "a batch needs at least one system");
  if (!offsets || !H || !pbc) throw Error(PFW_EINVAL, "offsets, cells and pbc are required");
  if (offsets[0] != 0) throw Error(PFW_EINVAL, "atom offsets must start at 0");
  for (int32_t s = 0; s < nsys; ++s)
    if (offsets[s + 1] < offsets[s]) throw Error(PFW_EINVAL, "atom offsets must be nondecreasing");
  const int64_t n = offsets[nsys];
  if (n > (int64_t)INT32_MAX / 4) throw Error(PFW_EINVAL, "atom count out of range");
  if (n > 0 && (!X || !species)) throw Error(PFW_EINVAL, "positions and species are required");
  std::vector<pfw::HostSystem> systems(nsys);
  for (int32_t s = 0; s < nsys; ++s) {
    pfw::HostSystem& hs = systems[s];
    for (int k = 0; k < 9; ++k) hs.H[k] = H[9 * (size_t)s + k];
    for (int a = 0; a < 3; ++a) hs.pbc[a] = pbc[3 * (size_t)s + a] ? 1 : 0;
    hs.atom_begin = (int32_t)offsets[s];
    hs.natoms = (int32_t)(offsets[s + 1] - offsets[s]);
  }
  int32_t max_species = 0;
  if (!device_ptrs)
    for (int64_t i = 0; i < n; ++i) {
      if (species[i] < 0) throw Error(PFW_EINVAL, "species channels must be nonnegative");
      max_species = std::max(max_species, species[i]);
    }
  cudaMemcpyKind kind = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  ws->X.ensure(sizeof(double) * 3 * std::max<int64_t>(n, 1));
  ws->species.ensure(sizeof(int32_t) * std::max<int64_t>(n, 1));
  if (n > 0) {
    PFW_CUDA(cudaMemcpyAsync(ws->X.ptr, X, sizeof(double) * 3 * n, kind, ws->stream));
    PFW_CUDA(cudaMemcpyAsync(ws->species.ptr, species, sizeof(int32_t) * n, kind, ws->stream));
  }
  ws->systems.swap(systems);
  ws->n = (int32_t)n;
  ws->n_owned = -1;
  ws->max_species = max_species;
  ws->geometry_version += 1;
  ws->prep.valid = false;
  ws->nb_total = -1;
  ws->last_pairs = -1;
}

void dispatch_evaluate(pfw_ws* ws, int32_t model, uint32_t request, double* E, double* F, double* W) {
  if (model == PFW_MODEL_PAIR) pfw::pair_evaluate(ws, request, E, F, W);
  else if (model == PFW_MODEL_ACE) pfw::ace_evaluate(ws, request, E, F, W);
  else if (model == PFW_MODEL_SURROGATE) pfw::sur_evaluate(ws, request, E, F, W);
  else throw Error(PFW_EINVAL, "unknown model selector");
  ws->last_model = model;
}

// Batch evaluation on device outputs (no host synchronisation for pairs).
void evaluate_batch_device(pfw_ws* ws, int32_t model, uint32_t request, double* E, double* F, double* W,
                           double* feat) {
  if (ws->systems.empty()) throw Error(PFW_ESTATE, "no geometry set");
  if (model == PFW_MODEL_PAIR) {
    if (feat) throw Error(PFW_EINVAL, "fitting features exist for ACE models only");
    pfw::pair_evaluate(ws, request, E, F, W, true);
  } else if (model == PFW_MODEL_ACE) {
    pfw::ace_evaluate_batch(ws, request, E, F, W, feat);
  } else {
    throw Error(PFW_EINVAL, "unknown model selector");
  }
}

}  // namespace

extern "C" {

const char* pfw_version(void) { return "0.1.0"; }

pfw_status pfw_ws_create(const pfw_options* opts, pfw_ws** out) {
  if (!out) return PFW_EINVAL;
  *out = nullptr;
  pfw_ws* ws = new (std::nothrow) pfw_ws();
  if (!ws) return PFW_ECUDA;
  if (opts) ws->opt = *opts;
  else {
    ws->opt.precision = PFW_PRECISION_FP64;
    ws->opt.bruteforce_threshold = 32;
    ws->opt.device = 0;
  }
  if (ws->opt.bruteforce_threshold < 0 ||
      (ws->opt.precision != PFW_PRECISION_FP64 && ws->opt.precision != PFW_PRECISION_MIXED)) {
    delete ws;
    return PFW_EINVAL;
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev <= ws->opt.device) {
    delete ws;
    return PFW_ECUDA;
  }
  if (cudaSetDevice(ws->opt.device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ws;
    return PFW_ECUDA;
  }
  ws->own_stream = ws->stream;
  *out = ws;
  return PFW_OK;
}

void pfw_ws_destroy(pfw_ws* ws) {
  if (!ws) return;
  cudaSetDevice(ws->opt.device);
  if (ws->stream) cudaStreamSynchronize(ws->stream);
  pfw::ace_free(ws);
  pfw::sur_free(ws);
  pfw::skin_free(ws);
  pfw::pair_graph_free(ws);
  pfw::mlp_scratch_free(ws);
  if (ws->flags_host) cudaFreeHost(ws->flags_host);
  pfw::DevBuf* bufs[] = {&ws->X, &ws->species, &ws->atom_sys, &ws->sysgeom, &ws->wrapped, &ws->bincoord,
                         &ws->wind, &ws->cellid, &ws->slot, &ws->cell_count, &ws->cell_start, &ws->cell_sys,
                         &ws->tmp_idx, &ws->perm, &ws->inverse, &ws->pos, &ws->pos32, &ws->scan_tmp,
                         &ws->minmax, &ws->slab_scratch, &ws->cellpart, &ws->out_E, &ws->out_F, &ws->out_W, &ws->out_feat, &ws->counters, &ws->red_partial, &ws->pair_slots,
                         &ws->nb_count, &ws->nb_offsets, &ws->nb_j, &ws->nb_S, &ws->nb_R};
  for (auto* b : bufs) b->release();
  for (auto& e : ws->ev)
    if (e) cudaEventDestroy(e);
  if (ws->own_stream) cudaStreamDestroy(ws->own_stream);
  delete ws;
}

const char* pfw_last_error(const pfw_ws* ws) { return ws ? ws->err.c_str() : "null workspace"; }

pfw_status pfw_set_geometry(pfw_ws* ws, int64_t n, const double* X, const double* H, const uint8_t pbc[3],
                            const int32_t* species) {
  return guarded(ws, [&] { upload_geometry(ws, n, X, H, pbc, species, false); });
}

pfw_status pfw_set_geometry_device(pfw_ws* ws, int64_t n, const double* X_dev, const double* H,
                                   const uint8_t pbc[3], const int32_t* species_dev) {
  return guarded(ws, [&] { upload_geometry(ws, n, X_dev, H, pbc, species_dev, true); });
}

pfw_status pfw_set_owned(pfw_ws* ws, int64_t n_owned) {
  return guarded(ws, [&] {
    if (ws->systems.size() != 1) throw Error(PFW_ESTATE, "owned atoms apply to a single-system geometry");
    if (n_owned < -1 || n_owned > ws->n) throw Error(PFW_EINVAL, "owned atom count out of range");
    ws->n_owned = (int32_t)n_owned;
  });
}

pfw_status pfw_slab_bands(pfw_ws* ws, int64_t n, const double* X_dev, const int32_t* species_dev,
                          const double frac_row[3], double lo, double hi, double d, const double shift_lower[3],
                          const double shift_upper[3], double* lower_dev, double* upper_dev, int32_t* counts_dev) {
  return guarded(ws, [&] {
    if (!frac_row || !shift_lower || !shift_upper) throw Error(PFW_EINVAL, "slab axis row and shifts required");
    pfw::slab_bands(ws, n, X_dev, species_dev, frac_row, lo, hi, d, shift_lower, shift_upper, lower_dev, upper_dev,
                    counts_dev);
  });
}

pfw_status pfw_pair_set_skin(pfw_ws* ws, double skin) {
  return guarded(ws, [&] {
    if (!(std::isfinite(skin) && skin >= 0.0)) throw Error(PFW_EINVAL, "skin must be finite and nonnegative (Å)");
    ws->skin = skin;
  });
}

pfw_status pfw_pair_skin_stats(pfw_ws* ws, int64_t* builds, int64_t* reuses) {
  return guarded(ws, [&] { pfw::skin_stats(ws, builds, reuses); });
}

pfw_status pfw_pair_model_smooth(pfw_ws* ws, int32_t nz, const double* A, double cutoff) {
  return guarded(ws, [&] {
    if (nz < 1 || nz > 4) throw Error(PFW_EINVAL, "SmoothPair supports 1 to 4 species channels");
    if (!A) throw Error(PFW_EINVAL, "amplitude table required");
    if (!(std::isfinite(cutoff) && cutoff > 0)) throw Error(PFW_EINVAL, "cutoff must be finite and positive");
    for (int a = 0; a < nz; ++a)
      for (int b = 0; b < nz; ++b)
        if (!std::isfinite(A[a * nz + b]) || A[a * nz + b] != A[b * nz + a])
          throw Error(PFW_EINVAL, "amplitude table must be finite and symmetric");
    const std::vector<double> amp(A, A + nz * nz);
    if (!(ws->pair.kind == 0 && ws->pair.nz == nz && ws->pair.A == amp && ws->pair.cutoff == cutoff))
      ws->model_version += 1;  // an unchanged model keeps captured evaluations valid
    ws->pair.kind = 0;
    ws->pair.nz = nz;
    ws->pair.A = amp;
    ws->pair.cutoff = cutoff;
  });
}

pfw_status pfw_pair_model_lj(pfw_ws* ws, double epsilon, double sigma, double cutoff) {
  return guarded(ws, [&] {
    if (!(std::isfinite(epsilon) && std::isfinite(sigma) && std::isfinite(cutoff) && epsilon > 0 && sigma > 0 &&
          cutoff > 0))
      throw Error(PFW_EINVAL, "LJ parameters must be positive and finite");
    if (!(ws->pair.kind == 1 && ws->pair.eps == epsilon && ws->pair.sigma == sigma && ws->pair.cutoff == cutoff))
      ws->model_version += 1;
    ws->pair.kind = 1;
    ws->pair.nz = 1;
    ws->pair.eps = epsilon;
    ws->pair.sigma = sigma;
    ws->pair.cutoff = cutoff;
  });
}

pfw_status pfw_ace_model_load(pfw_ws* ws, const pfw_ace_tables* tables) {
  return guarded(ws, [&] {
    if (!tables) throw Error(PFW_EINVAL, "tables required");
    pfw::ace_load(ws, tables);
  });
}

pfw_status pfw_ace_set_schedule(pfw_ws* ws, int32_t chunk, int32_t groups) {
  return guarded(ws, [&] { pfw::ace_set_schedule(ws, chunk, groups); });
}

pfw_status pfw_evaluate_device(pfw_ws* ws, int32_t model, uint32_t request, double* E_dev, double* F_dev,
                               double* W_dev) {
  return guarded(ws, [&] {
    if (ws->systems.empty()) throw Error(PFW_ESTATE, "no geometry set");
    dispatch_evaluate(ws, model, request, E_dev, F_dev, W_dev);
  });
}

pfw_status pfw_evaluate(pfw_ws* ws, int32_t model, uint32_t request, double* E, double* F, double* W) {
  return guarded(ws, [&] {
    if (ws->systems.empty()) throw Error(PFW_ESTATE, "no geometry set");
    const int n = ws->n;
    double* dE = static_cast<double*>(ws->out_E.ensure(sizeof(double)));
    double* dW = static_cast<double*>(ws->out_W.ensure(sizeof(double) * 9));
    double* dF = (request & PFW_REQ_FORCES) ? static_cast<double*>(ws->out_F.ensure(sizeof(double) * 3 * std::max(n, 1)))
                                            : nullptr;
    // the pair path's cell-list flags come back with the outputs (one synchronisation)
    ws->defer_check = model == PFW_MODEL_PAIR;
    ws->check_pending = false;
    try {
      dispatch_evaluate(ws, model, request, dE, dF, dW);
    } catch (...) {
      ws->defer_check = false;
      if (ws->check_pending) {
        ws->check_pending = false;
        cudaStreamSynchronize(ws->stream);
      }
      throw;
    }
    ws->defer_check = false;
    double hE = 0, hW[9];
    unsigned long long np = 0;
    PFW_CUDA(cudaMemcpyAsync(&hE, dE, sizeof(double), cudaMemcpyDeviceToHost, ws->stream));
    PFW_CUDA(cudaMemcpyAsync(hW, dW, sizeof(double) * 9, cudaMemcpyDeviceToHost, ws->stream));
    if (model == PFW_MODEL_PAIR)
      PFW_CUDA(cudaMemcpyAsync(&np, static_cast<unsigned long long*>(ws->counters.ptr) + 4, sizeof(np),
                               cudaMemcpyDeviceToHost, ws->stream));
    if (F && dF && n > 0)
      PFW_CUDA(cudaMemcpyAsync(F, dF, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, ws->stream));
    PFW_CUDA(cudaStreamSynchronize(ws->stream));
    pfw::prepare_check_finish(ws);
    if (model == PFW_MODEL_PAIR) ws->last_pairs = (int64_t)np / 2;
    // the reference GPU reports nonfinite results as a DomainError (NeighbourList/gpu.jl:391-395)
    bool finite = std::isfinite(hE);
    for (double v : hW) finite = finite && std::isfinite(v);
    if (!finite) throw Error(PFW_EDOMAIN, "nonfinite energy/virial (coincident atoms with a singular model?)");
    if (E) *E = hE;
    if (W)
      for (int k = 0; k < 9; ++k) W[k] = hW[k];
  });
}

pfw_status pfw_set_batch(pfw_ws* ws, int32_t nsys, const int64_t* atom_offsets, const double* X, const double* H,
                         const uint8_t* pbc, const int32_t* species) {
  return guarded(ws, [&] { upload_batch(ws, nsys, atom_offsets, X, H, pbc, species, false); });
}

pfw_status pfw_set_batch_device(pfw_ws* ws, int32_t nsys, const int64_t* atom_offsets, const double* X_dev,
                                const double* H, const uint8_t* pbc, const int32_t* species_dev) {
  return guarded(ws, [&] { upload_batch(ws, nsys, atom_offsets, X_dev, H, pbc, species_dev, true); });
}

pfw_status pfw_batch_update_positions(pfw_ws* ws, const double* X, int32_t on_device) {
  return guarded(ws, [&] {
    if (ws->systems.empty()) throw Error(PFW_ESTATE, "no geometry set");
    if (ws->n > 0 && !X) throw Error(PFW_EINVAL, "positions required");
    if (ws->n > 0)
      PFW_CUDA(cudaMemcpyAsync(ws->X.ptr, X, sizeof(double) * 3 * ws->n,
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ws->stream));
    if (!on_device) PFW_CUDA(cudaStreamSynchronize(ws->stream));
    ws->prep.valid = false;
    ws->nb_total = -1;
  });
}

pfw_status pfw_ace_feature_count(pfw_ws* ws, int32_t* nfeat) {
  return guarded(ws, [&] {
    if (!nfeat) throw Error(PFW_EINVAL, "null output");
    *nfeat = pfw::ace_feature_count(ws);
  });
}

pfw_status pfw_ace_design_shape(pfw_ws* ws, int64_t* rows, int64_t* cols) {
  return guarded(ws, [&] {
    if (ws->systems.empty()) throw Error(PFW_ESTATE, "no geometry set");
    pfw::ace_design_shape(ws, rows, cols);
  });
}

pfw_status pfw_ace_design_matrix_device(pfw_ws* ws, double* A_dev, int64_t ld, int64_t rows_capacity,
                                        double* baseline_dev) {
  return guarded(ws, [&] {
    if (ws->systems.empty()) throw Error(PFW_ESTATE, "no geometry set");
    pfw::ace_design_matrix(ws, A_dev, ld, rows_capacity, baseline_dev);
  });
}

pfw_status pfw_ace_design_matrix(pfw_ws* ws, double* A, int64_t ld, int64_t rows_capacity, double* baseline) {
  return guarded(ws, [&] {
    if (ws->systems.empty()) throw Error(PFW_ESTATE, "no geometry set");
    if (!A) throw Error(PFW_EINVAL, "null design matrix");
    int64_t rows = 0, cols = 0;
    pfw::ace_design_shape(ws, &rows, &cols);
    if (ld < cols || rows_capacity < rows) throw Error(PFW_ESHAPE, "design matrix buffer too small");
    const size_t nsys = ws->systems.size();
    double* dA = static_cast<double*>(ws->out_design.ensure(sizeof(double) * std::max<int64_t>(rows * cols, 1)));
    double* dB = static_cast<double*>(ws->out_base.ensure(sizeof(double) * std::max<size_t>(nsys, 1)));
    pfw::ace_design_matrix(ws, dA, cols, rows, dB);
    if (rows > 0 && cols > 0)
      PFW_CUDA(cudaMemcpy2DAsync(A, sizeof(double) * ld, dA, sizeof(double) * cols, sizeof(double) * cols, rows,
                                 cudaMemcpyDeviceToHost, ws->stream));
    if (baseline && nsys > 0)
      PFW_CUDA(cudaMemcpyAsync(baseline, dB, sizeof(double) * nsys, cudaMemcpyDeviceToHost, ws->stream));
    PFW_CUDA(cudaStreamSynchronize(ws->stream));
  });
}

pfw_status pfw_evaluate_batch_device(pfw_ws* ws, int32_t model, uint32_t request, double* E_dev, double* F_dev,
                                     double* W_dev, double* features_dev) {
  return guarded(ws, [&] {
    evaluate_batch_device(ws, model, request, E_dev, F_dev, W_dev, features_dev);
    PFW_CUDA(cudaStreamSynchronize(ws->stream));
    PFW_CUDA(cudaGetLastError());
  });
}

pfw_status pfw_evaluate_batch(pfw_ws* ws, int32_t model, uint32_t request, double* E, double* F, double* W,
                              double* features) {
  return guarded(ws, [&] {
    if (ws->systems.empty()) throw Error(PFW_ESTATE, "no geometry set");
    const int n = ws->n, nsys = (int)ws->systems.size();
    const int nfeat = (features && model == PFW_MODEL_ACE) ? pfw::ace_feature_count(ws) : 0;
    double* dE = static_cast<double*>(ws->out_E.ensure(sizeof(double) * nsys));
    double* dW = static_cast<double*>(ws->out_W.ensure(sizeof(double) * 9 * nsys));
    double* dF = (request & PFW_REQ_FORCES) ? static_cast<double*>(ws->out_F.ensure(sizeof(double) * 3 * std::max(n, 1)))
                                            : nullptr;
    double* dX = features ? static_cast<double*>(ws->out_feat.ensure(sizeof(double) * std::max(nfeat, 1) * nsys))
                          : nullptr;
    evaluate_batch_device(ws, model, request, dE, dF, dW, dX);
    std::vector<double> hE(nsys), hW(9 * (size_t)nsys);
    PFW_CUDA(cudaMemcpyAsync(hE.data(), dE, sizeof(double) * nsys, cudaMemcpyDeviceToHost, ws->stream));
    PFW_CUDA(cudaMemcpyAsync(hW.data(), dW, sizeof(double) * 9 * nsys, cudaMemcpyDeviceToHost, ws->stream));
    if (F && dF && n > 0)
      PFW_CUDA(cudaMemcpyAsync(F, dF, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, ws->stream));
    if (features && dX && nfeat > 0)
      PFW_CUDA(cudaMemcpyAsync(features, dX, sizeof(double) * nfeat * nsys, cudaMemcpyDeviceToHost, ws->stream));
    PFW_CUDA(cudaStreamSynchronize(ws->stream));
    bool finite = true;
    for (double v : hE) finite = finite && std::isfinite(v);
    for (double v : hW) finite = finite && std::isfinite(v);
    if (!finite) throw Error(PFW_EDOMAIN, "nonfinite energy/virial (coincident atoms with a singular model?)");
    if (E) std::copy(hE.begin(), hE.end(), E);
    if (W) std::copy(hW.begin(), hW.end(), W);
  });
}

pfw_status pfw_batch_graph_launch(pfw_ws* ws, uint32_t request, double* E_dev, double* F_dev, double* W_dev,
                                  double* features_dev) {
  return guarded(ws, [&] {
    if (ws->systems.empty()) throw Error(PFW_ESTATE, "no geometry set");
    pfw::ace_batch_graph(ws, request, E_dev, F_dev, W_dev, features_dev);
  });
}

pfw_status pfw_batch_graph_sync(pfw_ws* ws) {
  return guarded(ws, [&] { pfw::ace_batch_graph_sync(ws); });
}

pfw_status pfw_site_energies(pfw_ws* ws, double* energies) {
  return guarded(ws, [&] {
    if (ws->last_model == PFW_MODEL_SURROGATE) pfw::sur_site_energies(ws, energies);
    else pfw::ace_site_energies(ws, energies);
  });
}

pfw_status pfw_surrogate_load(pfw_ws* ws, const pfw_ace_tables* features, const pfw_mlp_params* mlp) {
  return guarded(ws, [&] {
    if (!features) throw Error(PFW_EINVAL, "feature model tables required");
    pfw::sur_load(ws, features, mlp);
  });
}

pfw_status pfw_surrogate_features(pfw_ws* ws, double* features) {
  return guarded(ws, [&] {
    if (ws->systems.empty()) throw Error(PFW_ESTATE, "no geometry set");
    if (!features) throw Error(PFW_EINVAL, "null output");
    int32_t nin = 0;
    pfw::sur_stats(ws, nullptr, nullptr);  // raises without a feature model
    nin = pfw::sur_feature_width(ws);
    double* d = static_cast<double*>(ws->out_feat.ensure(sizeof(double) * std::max<int64_t>(1, (int64_t)ws->n * nin)));
    pfw::sur_features(ws, d);
    if (ws->n > 0)
      PFW_CUDA(cudaMemcpyAsync(features, d, sizeof(double) * (size_t)ws->n * nin, cudaMemcpyDeviceToHost, ws->stream));
    PFW_CUDA(cudaStreamSynchronize(ws->stream));
  });
}

pfw_status pfw_surrogate_stats(pfw_ws* ws, int64_t* fallback_sites, int64_t* sites) {
  return guarded(ws, [&] { pfw::sur_stats(ws, fallback_sites, sites); });
}

pfw_status pfw_mlp_param_grad(pfw_ws* ws, const pfw_mlp_shape* shape, const float* params, int64_t n, const float* X,
                              const float* y, const int32_t* species, double* loss, float* grad) {
  return guarded(ws, [&] { pfw::mlp_param_grad(ws, shape, params, n, X, y, species, loss, grad); });
}

pfw_status pfw_mlp_ef_step(pfw_ws* ws, const pfw_mlp_shape* shape, float* params_dev, float* m1_dev, float* m2_dev,
                           int64_t n, const float* X_dev, const float* y_dev, const int32_t* species,
                           const float* V_dev, const float* c_dev, float wE, float lr, int64_t step, float* grad_dev,
                           double* loss) {
  return guarded(ws, [&] {
    pfw::mlp_ef_step(ws, shape, params_dev, m1_dev, m2_dev, n, X_dev, y_dev, species, V_dev, c_dev, wE, lr, step,
                     grad_dev, loss);
  });
}

pfw_status pfw_mlp_input_grad(pfw_ws* ws, const pfw_mlp_shape* shape, const float* params_dev, int64_t n,
                              const float* X_dev, const int32_t* species, float* G_dev) {
  return guarded(ws, [&] { pfw::mlp_input_grad(ws, shape, params_dev, n, X_dev, species, G_dev); });
}

pfw_status pfw_surrogate_pullback(pfw_ws* ws, const double* dEdx_dev, double* F_dev) {
  return guarded(ws, [&] { pfw::sur_pullback(ws, dEdx_dev, F_dev); });
}

pfw_status pfw_mlp_train(pfw_ws* ws, const pfw_mlp_shape* shape, float* params, int64_t n, const float* X,
                         const float* y, const int32_t* species, const pfw_mlp_train_options* options,
                         float* epoch_loss) {
  return guarded(ws, [&] { pfw::mlp_train(ws, shape, params, n, X, y, species, options, epoch_loss); });
}

pfw_status pfw_last_pair_count(pfw_ws* ws, int64_t* npairs) {
  return guarded(ws, [&] {
    if (!npairs) throw Error(PFW_EINVAL, "null output");
    *npairs = ws->last_pairs;
  });
}

pfw_status pfw_neighbour_count(pfw_ws* ws, double cutoff, int64_t* total) {
  return guarded(ws, [&] {
    ws->species_limit = INT32_MAX;  // the snapshot needs no model: any nonnegative channel
    int64_t t = pfw::neighbour_build(ws, cutoff);
    if (total) *total = t;
  });
}

pfw_status pfw_neighbour_fill(pfw_ws* ws, int64_t* offsets, int32_t* j, int32_t* S, double* R) {
  return guarded(ws, [&] { pfw::neighbour_fill(ws, offsets, j, S, R); });
}

pfw_status pfw_probe_fp64_peak(pfw_ws* ws, double* tflops) {
  return guarded(ws, [&] {
    double v = pfw::probe_fp64(ws);
    if (tflops) *tflops = v;
  });
}

uint64_t pfw_launch_count(const pfw_ws* ws) { return ws ? ws->launches : 0; }

pfw_status pfw_set_stream(pfw_ws* ws, void* stream) {
  return guarded(ws, [&] {
    PFW_CUDA(cudaStreamSynchronize(ws->stream));
    ws->stream = stream ? static_cast<cudaStream_t>(stream) : ws->own_stream;
  });
}

pfw_status pfw_set_diagnostics(pfw_ws* ws, int32_t on) {
  return guarded(ws, [&] {
    if (on && !ws->ev[0])
      for (auto& e : ws->ev) PFW_CUDA(cudaEventCreate(&e));
    ws->diag = on != 0;
    for (auto& u : ws->ev_used) u = false;
  });
}

int32_t pfw_stage_times(pfw_ws* ws, double* ms, int32_t cap) {
  if (!ws || !ws->diag || !ms) return 0;
  if (cudaSetDevice(ws->opt.device) != cudaSuccess) return 0;
  int32_t k = 0;
  for (int s = 0; s < 4 && k < cap; ++s, ++k) {
    float t = 0;
    if (ws->ev_used[s] && cudaEventSynchronize(ws->ev[2 * s + 1]) == cudaSuccess &&
        cudaEventElapsedTime(&t, ws->ev[2 * s], ws->ev[2 * s + 1]) == cudaSuccess)
      ms[k] = t;
    else
      ms[k] = 0;
  }
  return k;
}

}  // extern "C"
