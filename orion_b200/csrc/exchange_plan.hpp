// Exchange plan of one shard: which interface data stay inside the shard and
// which cross to another shard, derived from the global block list.
//
// Host-only (no CUDA), so it is unit-tested on the CPU.  Every shard computes
// the plan from the same global region lists in the same order, so the
// sender's and the receiver's lists for a pair of shards agree element for
// element without any negotiation; the wire order of a pair is the global
// (receiving block, region, point) order of the references.
//
// The two exchanges of a step:
// * exchange_bc (src/solver/HaloExchanger.cpp:70-179): each interface region of
//   a receiving block takes the 5 primitive components of its partner's sender
//   window (HaloExchanger.cpp:35-63).  Where windows of several regions cover
//   the same ghost element, the last region in the receiving block's file order
//   wins.  Pairs are (block, element) with element = m * npad + padded index.
// * average_interface_residuals (HaloExchanger.cpp:186-398): every interface
//   region packs dq/vol of its own points into slots; each receiving point then
//   averages, region by region, with the partner slots its image maps to.
//   A shard packs the slots of its own blocks; the slots of other shards that
//   its points read are received into an area after its own slots.
// With one shard (every owner 0) the plan is the single-case work list.
#pragma once
#include <algorithm>
#include <map>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "topology.hpp"

namespace orion {

struct ElemRef {
  int block;      // local block id
  long long elem; // m * npad + padded index of the block
};

struct ExchangePlan {
  int rank = 0;
  int nranks = 1;
  std::vector<int> local;     // global ids of the owned blocks, ascending; local id = position
  std::vector<int> local_of;  // global id -> local id, -1 if not owned
  // exchange_bc: destinations inside the shard with their final source
  std::vector<ElemRef> halo_dst, halo_src;
  std::vector<std::vector<ElemRef>> halo_send;  // per peer rank: own elements, wire order
  std::vector<std::vector<ElemRef>> halo_recv;  // per peer rank: own ghost elements, wire order
  // interface averaging
  std::vector<int> pk_block;        // own slots: local block and padded index
  std::vector<long long> pk_idx;
  std::vector<int> ap_block, ap_off{0}, ap_slot;  // receiving points, partner slots in region order
  std::vector<long long> ap_idx;
  std::vector<std::vector<int>> iface_send;  // per peer rank: own slots, wire order
  std::vector<int> iface_recv_base;          // per peer rank: first slot of its area
  std::vector<int> iface_recv_n;             // per peer rank: slots received
  int n_slots = 0;                           // own + received
};

// Builds the plan of shard `rank`; `owner` holds each global block's shard
// (empty: every block owned by shard 0).  Returns an empty string or the error.
inline std::string build_exchange_plan(const std::vector<HostBlock>& g, const std::vector<int>& owner_in, int rank,
                                       ExchangePlan& p, int ng) {
  const int nb = (int)g.size();
  std::vector<int> owner = owner_in.empty() ? std::vector<int>(nb, 0) : owner_in;
  if ((int)owner.size() != nb) return "owner list length differs from the block count";
  int nranks = 1;
  for (int o : owner) {
    if (o < 0) return "negative shard id";
    nranks = std::max(nranks, o + 1);
  }
  if (rank < 0 || rank >= nranks) return "rank outside the shards of the owner list";
  p = ExchangePlan();
  p.rank = rank;
  p.nranks = nranks;
  p.local_of.assign(nb, -1);
  for (int b = 0; b < nb; ++b)
    if (owner[b] == rank) {
      p.local_of[b] = (int)p.local.size();
      p.local.push_back(b);
    }
  p.halo_send.assign(nranks, {});
  p.halo_recv.assign(nranks, {});
  p.iface_send.assign(nranks, {});
  p.iface_recv_base.assign(nranks, 0);
  p.iface_recv_n.assign(nranks, 0);
  auto lin = [&](const HostBlock& h, int i, int j, int k) {
    return (long long)i + (long long)h.nx * ((long long)j + (long long)h.ny * k);
  };

  // ---------------- exchange_bc ----------------
  {
    struct Msg {
      int sb, tb, tw;
      std::vector<long long> src;  // elements of block sb
    };
    // A receiving block concerns this shard when the shard owns it or one of
    // its senders.  Every message to such a block is expanded: which sender
    // writes an element last depends on all of them.
    std::vector<char> concerns(nb, 0);
    for (int b = 0; b < nb; ++b) {
      if (owner[b] == rank) concerns[b] = 1;
      for (const auto& hr : g[b].regions) {
        const int tb = hr.r.nbt - 1;
        if (hr.r.nbt > 0 && tb < nb && owner[b] == rank) concerns[tb] = 1;
      }
    }
    std::vector<Msg> queue;
    for (int b = 0; b < nb; ++b) {
      const auto& h = g[b];
      const int dims[3] = {h.idim, h.jdim, h.kdim};
      for (const auto& hr : h.regions) {
        if (hr.r.nbt <= 0) continue;
        int beg[3], end[3];
        memory_window(hr, ng, dims, 0, beg, end);
        Msg msg{b, hr.r.nbt - 1, hr.r.ibcwin - 1, {}};
        if (msg.tb < nb && concerns[msg.tb])
          for (int m = 0; m < 5; ++m)
            for (int k = beg[2]; k <= end[2]; ++k)
              for (int j = beg[1]; j <= end[1]; ++j)
                for (int i = beg[0]; i <= end[0]; ++i) msg.src.push_back(m * h.npad + lin(h, i, j, k));
        queue.push_back(std::move(msg));
      }
    }
    {  // room for the pairs inside the shard: every owned ghost window, once
      size_t est = 0;
      for (int b = 0; b < nb; ++b) {
        if (owner[b] != rank) continue;
        const int dims[3] = {g[b].idim, g[b].jdim, g[b].kdim};
        for (const auto& hr : g[b].regions) {
          if (hr.r.nbt <= 0) continue;
          int beg[3], end[3];
          memory_window(hr, ng, dims, 1, beg, end);
          size_t n = 5;
          for (int d = 0; d < 3; ++d) n *= (size_t)std::max(0, end[d] - beg[d] + 1);
          est += n;
        }
      }
      p.halo_dst.reserve(est);
      p.halo_src.reserve(est);
    }
    std::vector<int> slot;
    std::vector<long long> dst, src_el;  // per receiving block, reused
    std::vector<int> src_blk;            // global block of each source element
    for (int b = 0; b < nb; ++b) {
      const auto& h = g[b];
      const int dims[3] = {h.idim, h.jdim, h.kdim};
      dst.clear();
      src_el.clear();
      src_blk.clear();
      if (concerns[b]) slot.assign((size_t)5 * h.npad, -1);
      for (int r = 0; r < (int)h.regions.size(); ++r) {
        const auto& hr = h.regions[r];
        if (hr.r.nbt <= 0) continue;
        auto it = std::find_if(queue.begin(), queue.end(), [&](const Msg& q) { return q.tb == b && q.tw == r; });
        if (it == queue.end())
          return "interface block " + std::to_string(b) + " region " + std::to_string(r) + " has no sending partner";
        if (concerns[b]) {
          int beg[3], end[3];
          memory_window(hr, ng, dims, 1, beg, end);
          std::vector<long long> pts;
          for (int k = beg[2]; k <= end[2]; ++k)
            for (int j = beg[1]; j <= end[1]; ++j)
              for (int i = beg[0]; i <= end[0]; ++i) pts.push_back(lin(h, i, j, k));
          const size_t np = pts.size();
          for (size_t q = 0; q < 5 * np && q < it->src.size(); ++q) {
            const long long el = (long long)(q / np) * h.npad + pts[q % np];
            int& sl = slot[(size_t)el];
            if (sl < 0) {
              sl = (int)dst.size();
              dst.push_back(el);
              src_blk.push_back(it->sb);
              src_el.push_back(it->src[q]);
            } else {
              src_blk[(size_t)sl] = it->sb;
              src_el[(size_t)sl] = it->src[q];
            }
          }
        }
        queue.erase(it);
      }
      const int ob = owner[b];
      for (size_t e = 0; e < dst.size(); ++e) {
        const int sb = src_blk[e], os = owner[sb];
        if (ob == rank && os == rank) {
          p.halo_dst.push_back({p.local_of[b], dst[e]});
          p.halo_src.push_back({p.local_of[sb], src_el[e]});
        } else if (ob == rank) {
          p.halo_recv[os].push_back({p.local_of[b], dst[e]});
        } else if (os == rank) {
          p.halo_send[ob].push_back({p.local_of[sb], src_el[e]});
        }
      }
    }
  }

  // ---------------- interface residual averaging ----------------
  {
    struct Src {
      int owner, base, n;  // the packing region's shard and its first slot there
    };
    std::map<std::pair<int, int>, Src> qsrc;  // target (block, region) -> packing region
    std::vector<int> nslot(nranks, 0);
    for (int b = 0; b < nb; ++b) {
      const auto& h = g[b];
      const int o = owner[b];
      for (int r = 0; r < (int)h.regions.size(); ++r) {
        const auto& gr = h.regions[r].r;
        if (gr.bctype >= 0) continue;
        int lo[3], hi[3];
        for (int d = 0; d < 3; ++d) {
          lo[d] = std::min(std::abs(gr.s_st[d]), std::abs(gr.s_ed[d]));
          hi[d] = std::max(std::abs(gr.s_st[d]), std::abs(gr.s_ed[d]));
        }
        Src s{o, nslot[o], 0};
        for (int k = lo[2]; k <= hi[2]; ++k)
          for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
              if (o == rank) {
                p.pk_block.push_back(p.local_of[b]);
                p.pk_idx.push_back(lin(h, i - 1 + ng, j - 1 + ng, k - 1 + ng));
              }
              s.n++;
            }
        nslot[o] += s.n;
        qsrc[{gr.nbt - 1, gr.ibcwin - 1}] = s;
      }
    }
    const int n_own = nslot[rank];
    // received slots: per source shard, first appearance of (shard, slot)
    std::vector<std::unordered_map<int, int>> recv_pos(nranks), send_pos(nranks);
    std::vector<int> ref_shard;  // per ap_slot entry: -1 own slot, else source shard (slot = position there)
    std::vector<int> eid;
    std::vector<std::vector<std::pair<int, int>>> eslots;  // per receiving point: (shard, slot)
    for (int b = 0; b < nb; ++b) {
      const auto& h = g[b];
      const int ob = owner[b];
      bool concerns = ob == rank;
      if (!concerns)
        for (int r = 0; r < (int)h.regions.size() && !concerns; ++r) {
          if (h.regions[r].r.bctype >= 0) continue;
          auto it = qsrc.find({b, r});
          if (it != qsrc.end() && it->second.owner == rank) concerns = true;
        }
      if (!concerns) {
        for (int r = 0; r < (int)h.regions.size(); ++r)
          if (h.regions[r].r.bctype < 0 && qsrc.find({b, r}) == qsrc.end())
            return "interface block " + std::to_string(b) + " region " + std::to_string(r) +
                   " receives no averaging data";
        continue;
      }
      eid.assign((size_t)h.npad, -1);
      eslots.clear();
      std::vector<long long> eidx;
      for (int r = 0; r < (int)h.regions.size(); ++r) {
        const auto& hr = h.regions[r];
        const auto& gr = hr.r;
        if (gr.bctype >= 0) continue;
        auto it = qsrc.find({b, r});
        if (it == qsrc.end())
          return "interface block " + std::to_string(b) + " region " + std::to_string(r) +
                 " receives no averaging data";
        std::vector<std::array<int, 3>> img;
        int md[3];
        interface_image(hr, img, md);
        int slo[3], tlo[3], thi[3];
        for (int d = 0; d < 3; ++d) {
          slo[d] = std::min(std::abs(gr.s_st[d]), std::abs(gr.s_ed[d]));
          tlo[d] = std::min(std::abs(gr.t_st[d]), std::abs(gr.t_ed[d]));
          thi[d] = std::max(std::abs(gr.t_st[d]), std::abs(gr.t_ed[d]));
        }
        const int nxt = thi[0] - tlo[0] + 1, nyt = thi[1] - tlo[1] + 1;
        for (int k = 0; k < md[2]; ++k)
          for (int j = 0; j < md[1]; ++j)
            for (int i = 0; i < md[0]; ++i) {
              const auto& t = img[(size_t)i + (size_t)md[0] * ((size_t)j + (size_t)md[1] * k)];
              const long long rem =
                  (long long)(t[0] - tlo[0]) + (long long)nxt * ((t[1] - tlo[1]) + (long long)nyt * (t[2] - tlo[2]));
              if (rem < 0 || rem >= it->second.n) return "interface averaging map leaves the partner window";
              const long long idx = lin(h, slo[0] + i - 1 + ng, slo[1] + j - 1 + ng, slo[2] + k - 1 + ng);
              int& e = eid[(size_t)idx];
              if (e < 0) {
                e = (int)eslots.size();
                eslots.emplace_back();
                eidx.push_back(idx);
              }
              eslots[(size_t)e].emplace_back(it->second.owner, it->second.base + (int)rem);
            }
      }
      for (size_t e = 0; e < eslots.size(); ++e) {
        if (ob == rank) {
          p.ap_block.push_back(p.local_of[b]);
          p.ap_idx.push_back(eidx[e]);
        }
        for (const auto& ref : eslots[e]) {
          const int os = ref.first, sl = ref.second;
          if (ob == rank) {
            if (os == rank) {
              p.ap_slot.push_back(sl);
              ref_shard.push_back(-1);
            } else {
              auto ins = recv_pos[os].emplace(sl, (int)recv_pos[os].size());
              p.ap_slot.push_back(ins.first->second);
              ref_shard.push_back(os);
            }
          } else if (os == rank) {
            auto ins = send_pos[ob].emplace(sl, (int)send_pos[ob].size());
            if (ins.second) p.iface_send[ob].push_back(sl);
          }
        }
        if (ob == rank) p.ap_off.push_back((int)p.ap_slot.size());
      }
    }
    int next = n_own;
    for (int s = 0; s < nranks; ++s) {
      p.iface_recv_base[s] = next;
      p.iface_recv_n[s] = (int)recv_pos[s].size();
      next += p.iface_recv_n[s];
    }
    for (size_t q = 0; q < p.ap_slot.size(); ++q)
      if (ref_shard[q] >= 0) p.ap_slot[q] += p.iface_recv_base[ref_shard[q]];
    p.n_slots = next;
  }
  return std::string();
}

}  // namespace orion
