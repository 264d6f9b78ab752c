// Device-side descriptors shared by the kernels and the host runtime.
#pragma once
#include <cstdint>

namespace orion {

constexpr int NG = 3;  // ghost layers (src/preprocess/FlowField.cpp:9-16)

// Scalar parameters (orion_params_t after conversion).
struct ParamsDev {
  double gamma, moo, reynolds, prl, cfl, twall, tref, visc;
  double roo, uoo, voo, woo, poo, too;
  double csrv;
  int nvis, method;
};

// One block's device arrays.  Every field is the reference's padded layout
// (i fastest, component slowest, component stride npad).  S is the storage
// type of the fields whose precision the mixed path lowers (dq, rhs, dt, c,
// mu, coed, node derivatives); prim, q, metrics and vol are always FP64.
template <typename S>
struct BlockDev {
  double* prim;           // 6 comps: rho,u,v,w,p,T
  double* q;              // 5 comps
  S* dq;                  // 5 comps
  const double* metrics;  // 9 comps
  const double* vol;
  S* dt;
  S* c;
  S* mu;
  S* duvwt;               // 12 comps: node derivatives of u,v,w,T along xi,eta,zeta
  const uint8_t* bcmask;  // 1 where a physical-BC window zeroes dq
  // FP32 shadows the mixed path's flux kernels read (nullptr on the plain path):
  // prim (6 comps) refreshed by the state kernel after the BCs, metrics (9) and
  // vol refreshed whenever they are set.  FP64 prim/metrics/vol stay the master.
  float* prim_f;
  float* met_f;
  float* vol_f;
  int ni, nj, nk;         // interior points
  int nx, ny, nz;         // padded
  long long npad;
  long long int_base;     // interior points of all earlier blocks (residual location key)

  // Plane-major ("skewed") copies of the implicit sweeps' operands.  Interior
  // points are ordered by hyperplane s = ii+jj+kk, then kk, then jj, so each
  // hyperplane is one contiguous range and a point's face neighbours lie in the
  // adjacent hyperplanes at offsets given by koff.  Component stride ncomp.
  int nplanes;            // ni + nj + nk - 2
  long long ncomp;        // ni * nj * nk
  const int* koff;        // start of run (s, kk) at koff[s * nk + kk]; koff[nplanes * nk] = ncomp
  const int* sk_nat;      // padded natural index of each compact point
  const int* sk_nb;       // 6 comps: compact index of the face neighbours (lower i,j,k, upper i,j,k), -1 outside
  S* sk_metrics;          // 9 comps (static)
  S* sk_vol;              // static
  S* sk_prim;             // 5 comps
  S* sk_mu;
  S* sk_coed;             // diagonal coefficient
  S* sk_rhs;              // 5 comps: masked RHS
  S* sk_dq;               // 5 comps: the increment being swept
  // Coefficients of the flux splitting that do not involve the swept increment
  // (computed once per step, off the sweeps' critical path):
  S* sk_nrm;              // 9 (static): unit normal nx_n,ny_n,nz_n of the point's xi, eta, zeta metrics
  S* sk_nbq;              // 8: u, v, w, H, c^2, (gamma-1)/2 v^2, c, 2 mu/(|Re| rho vol + 1e-30) of the point as
                          // somebody's neighbour
  S* sk_pair;             // 30: per face neighbour q (lower i,j,k, upper i,j,k): l1, x1, x2, ct_n, rv/2
  S* sk_gm;               // 3 (static): |grad xi|, |grad eta|, |grad zeta| of the point's metrics
  S* sk_inv;              // 3 (static): 1 / max(|grad .|, 1e-30)
  // the parameters of the block's case: kernels read them here, with the
  // block's other fields (no further dependent load), so one launch can
  // cover the blocks of several cases (orion_group_*)
  ParamsDev prm;
};

// A contiguous chunk of one block's points (padded or interior index space).
struct Chunk {
  int block;
  int count;
  long long start;
};

// A tile of whole grid lines of one block along one direction.
struct LineTile {
  int block;
  int first;  // first line id (lines enumerate the two transverse interior coordinates)
  int count;  // lines in the tile
  int pad;
};

// One physical BC region, memory coordinates (ghost offset applied).
struct RegionDev {
  int block;
  int type;
  int dir;      // 0,1,2
  int lr;       // +1 max face, otherwise min face
  int s_nd;     // 1-based normal direction
  int lo[3];    // inclusive window, memory coordinates
  int hi[3];
  int npts;
  int is2d;     // symmetry in a k-thin block
};

// Wavefront plane work: for plane s of a block, jj,kk of the line set.
struct PlaneChunk {
  int block;
  int start;  // first (jj + nj*kk) index
  int count;
  int pad;
};

// Residual partial of one CTA.
struct ResPartial {
  double sum;
  double max;
  long long key;  // lexicographic (block order, k, j, i, m) of the max
};

struct ResidualOut {
  double rms;
  double max;
  int loc[5];
  int pad;
  double phydtime;
};

// One case of a group stepped together: where its blocks, its chunks'
// partial results and its result slots are.
struct GroupMember {
  const void* blocks;            // the case's block descriptors in the group's array
  int nblocks;
  int part_off, part_n;          // its interior chunks (residual partials)
  int pad_off, pad_n;            // its padded chunks (time-step minima)
  long long total_points;        // interior points x 5
  unsigned long long* dtmin;     // the case's phydtime slot
  ResidualOut* hist;             // the case's history ring
  int* counter;
  ResPartial* total;
  // the case's own halo copy list (element indices into its arena)
  double* arena;
  const long long* halo_src;
  const long long* halo_dst;
  int n_halo;
};

}  // namespace orion
