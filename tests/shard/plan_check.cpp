// Host check of the shard exchange plan (orion_b200/csrc/exchange_plan.hpp).
//
// Reads a global block list and owner maps on stdin, then for every map
// emulates the two exchanges of a step on seeded arrays, once with the
// one-shard plan (the single-case work lists) and once shard by shard with
// explicit pack -> wire -> unpack between every pair, and requires the two to
// agree bit for bit on every block:
// * exchange_bc: ghost[dst] = state[src] for every pair;
// * average_interface_residuals: slots dq/vol packed first, then every
//   receiving point averaged with its partner slots in order.
// Also requires the sender's and receiver's list lengths of every pair to match.
//
// stdin:  nblocks
//         per block: idim jdim kdim nregions, then per region
//                    s_st[3] s_ed[3] t_st[3] t_ed[3] bctype nbt ibcwin
//         nmaps, then per map nblocks owner ids
// stdout: one line per map; exit status 1 on the first mismatch.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <vector>

#include "exchange_plan.hpp"

using namespace orion;

namespace {

constexpr int kNg = 3;

struct Rng {
  uint64_t s;
  double next() {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    return (double)(s >> 11) * (1.0 / 9007199254740992.0);
  }
};

bool same(const std::vector<double>& a, const std::vector<double>& b) {
  return a.size() == b.size() && std::memcmp(a.data(), b.data(), a.size() * sizeof(double)) == 0;
}

// exchange_bc through one plan per shard; state[g] is global block g's 5*npad elements
int check_halo(const std::vector<HostBlock>& g, const std::vector<ExchangePlan>& plans,
               const std::vector<std::vector<double>>& init, std::vector<std::vector<double>>& out) {
  out = init;
  const int nr = (int)plans.size();
  for (int r = 0; r < nr; ++r) {
    const auto& p = plans[r];
    for (size_t q = 0; q < p.halo_dst.size(); ++q) {
      const auto& d = p.halo_dst[q];
      const auto& s = p.halo_src[q];
      out[p.local[d.block]][d.elem] = init[p.local[s.block]][s.elem];
    }
  }
  for (int r = 0; r < nr; ++r)
    for (int s = 0; s < nr; ++s) {
      if (r == s) continue;
      const auto& snd = plans[r].halo_send[s];
      const auto& rcv = plans[s].halo_recv[r];
      if (snd.size() != rcv.size()) {
        std::printf("halo %d->%d: sends %zu, receiver expects %zu\n", r, s, snd.size(), rcv.size());
        return 1;
      }
      std::vector<double> wire;
      for (const auto& e : snd) wire.push_back(init[plans[r].local[e.block]][e.elem]);
      for (size_t i = 0; i < rcv.size(); ++i) out[plans[s].local[rcv[i].block]][rcv[i].elem] = wire[i];
    }
  (void)g;
  return 0;
}

int check_iface(const std::vector<HostBlock>& g, const std::vector<ExchangePlan>& plans,
                const std::vector<std::vector<double>>& dq0, const std::vector<std::vector<double>>& vol,
                std::vector<std::vector<double>>& dq) {
  dq = dq0;
  const int nr = (int)plans.size();
  std::vector<std::vector<double>> pack(nr);
  for (int r = 0; r < nr; ++r) {
    const auto& p = plans[r];
    pack[r].assign((size_t)p.n_slots * 5, std::nan(""));
    for (size_t t = 0; t < p.pk_block.size(); ++t) {
      const int gb = p.local[p.pk_block[t]];
      const long long idx = p.pk_idx[t];
      for (int m = 0; m < 5; ++m) pack[r][t * 5 + m] = dq0[gb][m * g[gb].npad + idx] / vol[gb][idx];
    }
  }
  for (int r = 0; r < nr; ++r)
    for (int s = 0; s < nr; ++s) {
      if (r == s) continue;
      const auto& snd = plans[r].iface_send[s];
      if ((int)snd.size() != plans[s].iface_recv_n[r]) {
        std::printf("iface %d->%d: sends %zu slots, receiver expects %d\n", r, s, snd.size(), plans[s].iface_recv_n[r]);
        return 1;
      }
      const int base = plans[s].iface_recv_base[r];
      for (size_t i = 0; i < snd.size(); ++i)
        for (int m = 0; m < 5; ++m) pack[s][(base + i) * 5 + m] = pack[r][(size_t)snd[i] * 5 + m];
    }
  for (int r = 0; r < nr; ++r) {
    const auto& p = plans[r];
    for (size_t e = 0; e < p.ap_block.size(); ++e) {
      const int gb = p.local[p.ap_block[e]];
      const long long idx = p.ap_idx[e];
      const double vs = vol[gb][idx];
      double q[5];
      for (int m = 0; m < 5; ++m) q[m] = dq0[gb][m * g[gb].npad + idx];
      for (int k = p.ap_off[e]; k < p.ap_off[e + 1]; ++k)
        for (int m = 0; m < 5; ++m) q[m] = 0.5 * (pack[r][(size_t)p.ap_slot[k] * 5 + m] * vs + q[m]);
      for (int m = 0; m < 5; ++m) dq[gb][m * g[gb].npad + idx] = q[m];
    }
  }
  return 0;
}

}  // namespace

int main() {
  int nb = 0;
  if (!(std::cin >> nb) || nb <= 0) return 2;
  std::vector<HostBlock> g(nb);
  for (int b = 0; b < nb; ++b) {
    int nreg = 0;
    std::cin >> g[b].idim >> g[b].jdim >> g[b].kdim >> nreg;
    g[b].nx = g[b].idim + 2 * kNg;
    g[b].ny = g[b].jdim + 2 * kNg;
    g[b].nz = g[b].kdim + 2 * kNg;
    g[b].npad = (long long)g[b].nx * g[b].ny * g[b].nz;
    const int dims[3] = {g[b].idim, g[b].jdim, g[b].kdim};
    for (int r = 0; r < nreg; ++r) {
      HostRegion hr{};
      auto& x = hr.r;
      for (int d = 0; d < 3; ++d) std::cin >> x.s_st[d];
      for (int d = 0; d < 3; ++d) std::cin >> x.s_ed[d];
      for (int d = 0; d < 3; ++d) std::cin >> x.t_st[d];
      for (int d = 0; d < 3; ++d) std::cin >> x.t_ed[d];
      std::cin >> x.bctype >> x.nbt >> x.ibcwin;
      classify_region(hr, dims);
      g[b].regions.push_back(hr);
    }
  }
  Rng rng{12345};
  std::vector<std::vector<double>> state(nb), dq(nb), vol(nb);
  for (int b = 0; b < nb; ++b) {
    state[b].resize((size_t)5 * g[b].npad);
    dq[b].resize((size_t)5 * g[b].npad);
    vol[b].resize((size_t)g[b].npad);
    for (auto& v : state[b]) v = rng.next();
    for (auto& v : dq[b]) v = rng.next() - 0.5;
    for (auto& v : vol[b]) v = 0.5 + rng.next();
  }
  ExchangePlan one;
  std::string err = build_exchange_plan(g, {}, 0, one, kNg);
  if (!err.empty()) {
    std::printf("one-shard plan: %s\n", err.c_str());
    return 1;
  }
  std::vector<std::vector<double>> halo1, avg1;
  check_halo(g, {one}, state, halo1);
  check_iface(g, {one}, dq, vol, avg1);

  int nmaps = 0;
  std::cin >> nmaps;
  for (int mi = 0; mi < nmaps; ++mi) {
    std::vector<int> owner(nb);
    int nr = 1;
    for (int b = 0; b < nb; ++b) {
      std::cin >> owner[b];
      nr = std::max(nr, owner[b] + 1);
    }
    std::vector<ExchangePlan> plans(nr);
    long long wire_halo = 0, wire_iface = 0;
    for (int r = 0; r < nr; ++r) {
      err = build_exchange_plan(g, owner, r, plans[r], kNg);
      if (!err.empty()) {
        std::printf("map %d shard %d: %s\n", mi, r, err.c_str());
        return 1;
      }
      for (const auto& v : plans[r].halo_send) wire_halo += (long long)v.size();
      for (const auto& v : plans[r].iface_send) wire_iface += 5 * (long long)v.size();
    }
    std::vector<std::vector<double>> halo, avg;
    if (check_halo(g, plans, state, halo) || check_iface(g, plans, dq, vol, avg)) return 1;
    for (int b = 0; b < nb; ++b) {
      if (!same(halo[b], halo1[b])) {
        std::printf("map %d: exchange_bc differs on block %d\n", mi, b);
        return 1;
      }
      if (!same(avg[b], avg1[b])) {
        std::printf("map %d: averaging differs on block %d\n", mi, b);
        return 1;
      }
    }
    std::printf("map %d: %d shards, identical; wire doubles halo %lld iface %lld\n", mi, nr, wire_halo, wire_iface);
  }
  return 0;
}
