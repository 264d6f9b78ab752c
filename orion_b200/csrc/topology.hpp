// Host-side topology: the work lists the kernels consume, derived from the
// region lists exactly as the reference derives its communication windows.
#pragma once
#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "orion_gpu.h"

namespace orion {

struct HostRegion {
  orion_region_t r;
  int s_nd = 0;  // 1..3 (BCReader.cpp:126-146)
  int s_lr = 0;  // -1 min, +1 max, 0 cut
};

struct HostBlock {
  int idim, jdim, kdim;
  int nx, ny, nz;
  long long npad;
  std::vector<HostRegion> regions;
};

// s_nd / s_lr as BCReader::read_parallel_bc_root_only computes them (BCReader.cpp:126-146).
inline void classify_region(HostRegion& hr, const int dims[3]) {
  const auto& r = hr.r;
  hr.s_nd = 0;
  hr.s_lr = 0;
  for (int d = 0; d < 3; ++d) {
    if (r.s_st[d] == r.s_ed[d]) {
      hr.s_nd = d + 1;
      if (r.s_st[d] == 1) hr.s_lr = -1;
      else if (r.s_st[d] == dims[d]) hr.s_lr = 1;
      else hr.s_lr = 0;
      break;
    }
  }
}

// get_memory_window (HaloExchanger.cpp:17-64): mode 0 = sender (interface
// plane and ng-1 planes inward), mode 1 = receiver (the ng ghost planes);
// tangentially widened by one point inside the block.
inline void memory_window(const HostRegion& hr, int ng, const int dims[3], int mode, int beg[3], int end[3]) {
  const auto& r = hr.r;
  int cc[3];
  for (int m = 0; m < 3; ++m) cc[m] = std::abs(r.s_st[m]) - 1 + ng;
  const int dir = hr.s_nd - 1;
  if (mode == 0) {
    if (hr.s_lr == -1) { beg[dir] = cc[dir]; end[dir] = cc[dir] + ng - 1; }
    else { beg[dir] = cc[dir] - ng + 1; end[dir] = cc[dir]; }
  } else {
    if (hr.s_lr == -1) { beg[dir] = cc[dir] - ng; end[dir] = cc[dir] - 1; }
    else { beg[dir] = cc[dir] + 1; end[dir] = cc[dir] + ng; }
  }
  for (int m = 0; m < 3; ++m) {
    if (m == dir) continue;
    int ps = std::min(std::abs(r.s_st[m]), std::abs(r.s_ed[m]));
    int pe = std::max(std::abs(r.s_st[m]), std::abs(r.s_ed[m]));
    if (ps > 1) ps -= 1;
    if (pe < dims[m]) pe += 1;
    beg[m] = ps - 1 + ng;
    end[m] = pe - 1 + ng;
  }
}

// Target coordinates of every point of an interface's source window, 1-based in
// the target block, flat index (i fastest) over the min..max window: the
// image/jmage/kmage maps of analyze_bc_connect (BCPreprocess.cpp:16-192).
inline void interface_image(const HostRegion& hr, std::vector<std::array<int, 3>>& img, int map_dims[3]) {
  const auto& r = hr.r;
  const int* s_st = r.s_st;
  const int* s_ed = r.s_ed;
  const int* t_st = r.t_st;
  const int* t_ed = r.t_ed;
  const int s_nd = hr.s_nd;
  int t_nd = 0;
  for (int m = 0; m < 3; ++m)
    if (t_st[m] == t_ed[m]) t_nd = m + 1;
  int dirm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // [t index][s index]
  bool done = false;
  for (int m = 0; m < 3 && !done; ++m) {
    for (int n = 0; n < 3 && !done; ++n) {
      if ((m + 1) != s_nd && (n + 1) != t_nd) {
        int js1 = s_st[m];
        if (std::abs(js1) < std::abs(s_ed[m])) js1 = s_ed[m];
        int js2 = t_st[n];
        if (std::abs(js2) < std::abs(t_ed[n])) js2 = t_ed[n];
        if (js1 * js2 > 0) {
          dirm[n][m] = 1;
          dirm[t_nd - 1][s_nd - 1] = 1;
          const int rem_t = 6 - (n + 1) - t_nd;
          const int rem_s = 6 - (m + 1) - s_nd;
          dirm[rem_t - 1][rem_s - 1] = 1;
          done = true;
        }
      }
    }
  }
  int s_sign[3], t_sign[3], st_sign[3];
  for (int m = 0; m < 3; ++m) {
    s_sign[m] = 1;
    if ((m + 1) != s_nd && std::abs(s_st[m]) > std::abs(s_ed[m])) s_sign[m] = -1;
    t_sign[m] = 1;
    if ((m + 1) != t_nd && std::abs(t_st[m]) > std::abs(t_ed[m])) t_sign[m] = -1;
  }
  for (int m = 0; m < 3; ++m) {
    int co = 0;
    for (int n = 0; n < 3; ++n)
      if (dirm[n][m] == 1) co = n;
    st_sign[m] = t_sign[co] * s_sign[m];
  }
  int lo[3], hi[3];
  for (int m = 0; m < 3; ++m) {
    lo[m] = std::min(std::abs(s_st[m]), std::abs(s_ed[m]));
    hi[m] = std::max(std::abs(s_st[m]), std::abs(s_ed[m]));
    map_dims[m] = hi[m] - lo[m] + 1;
  }
  img.assign((size_t)map_dims[0] * map_dims[1] * map_dims[2], {0, 0, 0});
  for (int k = std::abs(s_st[2]); k != std::abs(s_ed[2]) + s_sign[2]; k += s_sign[2])
    for (int j = std::abs(s_st[1]); j != std::abs(s_ed[1]) + s_sign[1]; j += s_sign[1])
      for (int i = std::abs(s_st[0]); i != std::abs(s_ed[0]) + s_sign[0]; i += s_sign[0]) {
        const int idelt = (i - std::abs(s_st[0])) * st_sign[0];
        const int jdelt = (j - std::abs(s_st[1])) * st_sign[1];
        const int kdelt = (k - std::abs(s_st[2])) * st_sign[2];
        std::array<int, 3> v;
        for (int n = 0; n < 3; ++n)
          v[n] = std::abs(t_st[n]) + dirm[n][0] * idelt + dirm[n][1] * jdelt + dirm[n][2] * kdelt;
        const size_t flat =
            (size_t)(i - lo[0]) + (size_t)map_dims[0] * ((size_t)(j - lo[1]) + (size_t)map_dims[1] * (size_t)(k - lo[2]));
        img[flat] = v;
      }
}

}  // namespace orion
