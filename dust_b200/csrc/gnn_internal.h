// gnn_internal.h -- learned preconditioner handle and shared entry points.
#pragma once

#include <cublas_v2.h>

#include <vector>

#include "dust_common.cuh"
#include "fmm_internal.h"

#define PC_FIN 8    // node input features
#define PC_EF 4     // edge features
#define PC_H 64     // hidden width
#define PC_L 3      // message-passing layers
#define PC_C 8      // training columns: 7 probe vectors + the solution
#define PC_KMAX 33  // neighbours + self
#define PC_NPAR (PC_H * PC_FIN + PC_H + PC_L * (2 * PC_H * PC_H + PC_H) + PC_H + PC_EF)

struct PcSample {
  DevBuf x, ef, w, Y, T;
};

struct dust_precond {
  int n = 0, K = 0;  // nodes, neighbour slots per node (slot 0 = self)
  cudaStream_t st = nullptr;
  cublasHandle_t cb = nullptr;
  DevBuf nbr, dist;              // [n][K] neighbour index, distance
  DevBuf par, grad, am, av;      // weights, gradient, Adam moments
  int adam_t = 0;
  std::vector<PcSample> samples;
  DevBuf h, z, m, dh, dhp, dm;   // activations and their gradients
  DevBuf o, R, loss;             // edge outputs, residual columns, loss + stats
  DevBuf ix, ief, iw, dinv;      // inference inputs of the current system
  DevBuf tmp;
};

// read-only view of an assembled system: the static block from its
// unfactored copy As (nst x nst), everything else from A (n x n)
struct SysView {
  int n, nst;
  const double *As, *A;
};

int pc_infer(dust_precond *p, const SysView &sv);
void pc_apply(dust_precond *p, const double *v, double *y, cudaStream_t st);
int pc_pack_sample(int n, int C, const double *dinv, const double *AZ, const double *Z,
                   const double *b, const double *x, float *Y, float *T, cudaStream_t st);
