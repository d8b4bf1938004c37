// ace.cu — ACE site energy, force and virial (placeholder until the site
// kernels land) and the FP64 throughput probe.
#include "pfw_internal.h"

namespace pfw {

struct AceDevice {};

void ace_load(pfw_ws*, const pfw_ace_tables*) { throw Error(PFW_ESTATE, "ACE kernels not available in this build"); }
void ace_free(pfw_ws* ws) {
  delete ws->ace;
  ws->ace = nullptr;
}
void ace_evaluate(pfw_ws*, uint32_t, double*, double*, double*) { throw Error(PFW_ESTATE, "no ACE model loaded"); }
void ace_site_energies(pfw_ws*, double*) { throw Error(PFW_ESTATE, "no ACE model loaded"); }

// FP64 FMA throughput: 8 independent dependency chains per thread.
__global__ void k_fp64_probe(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-3 + k;
  for (int it = 0; it < iters; ++it)
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == 1.2345) out[0] = s;  // keep the chains live
}

double probe_fp64(pfw_ws* ws) {
  int sms = 0;
  PFW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ws->opt.device));
  double* out = static_cast<double*>(ws->out_E.ensure(sizeof(double)));
  const int blocks = sms * 8, threads = 256, iters = 4096;
  cudaEvent_t e0, e1;
  PFW_CUDA(cudaEventCreate(&e0));
  PFW_CUDA(cudaEventCreate(&e1));
  k_fp64_probe<<<blocks, threads, 0, ws->stream>>>(out, 64, 0.999999, 1e-7);  // warm-up
  PFW_CUDA(cudaEventRecord(e0, ws->stream));
  k_fp64_probe<<<blocks, threads, 0, ws->stream>>>(out, iters, 0.999999, 1e-7);
  PFW_CUDA(cudaEventRecord(e1, ws->stream));
  PFW_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  PFW_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ws->launches += 2;
  double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
  return flops / (ms * 1e-3) / 1e12;
}

}  // namespace pfw
