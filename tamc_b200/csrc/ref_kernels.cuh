// ref_kernels.cuh -- argument blocks and launchers of the reference-order kernels.
#pragma once
#include "device.cuh"

namespace tamc {

struct RefInst {  // reference-order CSR (device pointers)
  uint32_t n;
  float offset;
  const uint32_t* rp;
  const uint32_t* col;
  const float* J;
  const float* bias;
  uint32_t g_nodes;
  const uint32_t* grp;
  const uint32_t* gcol;
  const double* sus;
};

struct RefPt {  // replica state of one PT run (device pointers)
  int8_t* spins;    // [R][n], replica-major
  float* energy;    // [R] cached f32 energies
  uint32_t* perm;   // [C][nt] slot -> replica
  uint8_t* tags;    // [C][nt]
  uint32_t* acc;    // [C][nt]
  uint32_t* rtrips; // [C]
  uint32_t* dhist;  // [C][nt][2]
  float* e_stale;   // [C][nt] scratch
  const float* betas;
  const float* dbeta;
  uint32_t nt, C, lo;
  uint32_t* visited;  // scratch [max(n, 1)]
  uint32_t* queue;    // scratch [max(n, 1)]
  float* rows;        // scratch [max(n, 1)]
};

struct MeasOut {  // PtIcmThermalSamples buffers on the device
  uint32_t M, S, nchi, level;
  float* e;        // [nt][M*C]
  int32_t* q;      // [nt][M*C/2]
  float* sus;      // [nt][nchi][M*C/2]
  uint8_t* samp;   // [Z][S*C][ceil(n/8)]
};

struct GsLog {  // ground-state trajectory ring for one run
  uint32_t cap;
  uint32_t* count;
  int* have;
  float* minE;
  uint32_t* steps;
  float* E;
  uint64_t* words;  // [cap][ceil(n/64)]
};

RefInst make_ref_inst(const tamc_inst* d);
void ref_energy_all(cudaStream_t st, const RefInst& I, const int8_t* spins, float* energy, uint32_t R);
void ref_icm(cudaStream_t st, const RefInst& I, const RefPt& P, const ExpTable& X, Xo* rng, int* err);
void ref_exchange_threaded(cudaStream_t st, const RefPt& P, const ExpTable& X, Xo* rngs);
void ref_sweep_threaded(cudaStream_t st, const RefInst& I, const RefPt& P, const ExpTable& X, Xo* rngs);
void ref_serial_round(cudaStream_t st, const RefInst& I, const RefPt& P, const ExpTable& X, Xo* rng);
void ref_measure(cudaStream_t st, const RefInst& I, const RefPt& P, const MeasOut& O, uint32_t m, bool meas,
                 uint32_t smp, bool samp);
void ref_gs_track(cudaStream_t st, const RefInst& I, const RefPt& P, const GsLog& L, uint32_t step);
void ref_sa(cudaStream_t st, const RefInst& I, const ExpTable& X, int8_t* spins, Xo* rngs, uint32_t parts,
            uint32_t per, const float* betas, uint32_t nbeta);

}  // namespace tamc
