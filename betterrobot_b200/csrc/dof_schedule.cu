// dof_schedule.cu — host-side builder of the level schedule that the LM kernel uses to
// factor J^T J + damp I over the DOF tree (br_tree_t.dof_sched; layout in br_b200.h).
//
// The reference solves each LM step with a dense Cholesky of the full nv x nv normal
// matrix (src/better_robot/optim/optimizers/levenberg_marquardt.py:95-97 through
// optim/solvers/cholesky.py:14-18).  J^T J of a kinematic tree is sparse: columns c and c'
// interact only when one is an ancestor of the other in the DOF tree, so eliminating
// leaves first creates no fill-in.  This file lays that elimination out in levels of
// independent DOFs so that one team of lanes runs a whole level between two
// synchronisations (13 levels instead of 36 pivots for a floating-base humanoid).
#include <stdint.h>

#include <algorithm>
#include <unordered_map>
#include <vector>

#include "../../include/br_b200.h"

namespace {

struct Contrib {
  uint32_t a, b, d;
};

}  // namespace

extern "C" int64_t br_dof_schedule(const int32_t* dof_parent, int32_t nv, uint32_t* out, int64_t capacity) {
  if (nv < 0 || nv > BR_MAX_NV || (nv > 0 && !dof_parent) || capacity < 0) return BR_EINVAL;
  std::vector<int> dep(nv), rowoff(nv + 1), height(nv, 0);
  std::vector<std::vector<int>> anc(nv);  // ancestors of c by depth (root first)
  int nl = 0;
  for (int c = 0; c < nv; ++c) {
    const int p = dof_parent[c];
    if (p < -1 || p >= c) return BR_EINVAL;
    dep[c] = p < 0 ? 0 : dep[p] + 1;
    if (p >= 0) {
      anc[c] = anc[p];
      anc[c].push_back(p);
    }
    rowoff[c] = nl;
    nl += dep[c] + 1;
  }
  rowoff[nv] = nl;
  if (nl + nv > 0xffff) return BR_ETOOBIG;
  for (int c = nv - 1; c >= 0; --c)
    if (dof_parent[c] >= 0) height[dof_parent[c]] = std::max(height[dof_parent[c]], height[c] + 1);
  int levels = 0, depth_levels = 0;
  for (int c = 0; c < nv; ++c) {
    levels = std::max(levels, height[c] + 1);
    depth_levels = std::max(depth_levels, dep[c] + 1);
  }
  const uint32_t zoff = (uint32_t)nl;  // right-hand-side slots follow the packed rows

  std::vector<uint32_t> starts;
  std::vector<uint32_t> tasks;   // 4 words each
  std::vector<uint32_t> extras;  // 2 words each
  for (int lev = 0; lev < levels; ++lev) {
    starts.push_back((uint32_t)(tasks.size() / 4));
    std::vector<std::pair<uint32_t, std::vector<Contrib>>> groups;
    std::unordered_map<uint32_t, size_t> where;
    auto add = [&](uint32_t dst, Contrib c) {
      auto it = where.find(dst);
      if (it == where.end()) {
        where.emplace(dst, groups.size());
        groups.push_back({dst, {c}});
      } else {
        groups[it->second].second.push_back(c);
      }
    };
    for (int k = nv - 1; k >= 0; --k) {  // descending DOF index: the one-at-a-time order
      if (height[k] != lev) continue;
      const uint32_t rk = (uint32_t)rowoff[k], d = (uint32_t)k;
      for (int a = 0; a < dep[k]; ++a)
        for (int b = 0; b <= a; ++b) add((uint32_t)(rowoff[anc[k][a]] + b), {rk + a, rk + b, d});
      for (int a = 0; a < dep[k]; ++a) add(zoff + (uint32_t)anc[k][a], {rk + a, zoff + (uint32_t)k, d});
    }
    // entries with several contributions first, so that they spread over the lanes
    std::stable_sort(groups.begin(), groups.end(),
                     [](const auto& x, const auto& y) { return x.second.size() > y.second.size(); });
    for (const auto& g : groups) {
      const uint32_t n_extra = (uint32_t)g.second.size() - 1, first = (uint32_t)(extras.size() / 2);
      if (n_extra > 0xffff || first + n_extra > 0xffff) return BR_ETOOBIG;
      const Contrib& c0 = g.second[0];
      tasks.insert(tasks.end(), {g.first | (n_extra << 16), c0.a | (c0.b << 16), c0.d | (first << 16), 0u});
      for (size_t e = 1; e < g.second.size(); ++e) {
        const Contrib& c = g.second[e];
        extras.insert(extras.end(), {c.a | (c.b << 16), c.d});
      }
    }
  }
  const uint32_t n_tasks = (uint32_t)(tasks.size() / 4);
  starts.push_back(n_tasks);
  // the last task that updates DOF k's diagonal finalises its pivot: flag it (word 3 = k + 1)
  // so that the lane running it also stores 1 / (pivot + damp) for the levels above
  std::vector<int64_t> last(nv, -1);
  for (uint32_t p = 0; p < n_tasks; ++p) {
    const int dst = (int)(tasks[4 * p] & 0xffff);
    if (dst >= nl) continue;
    const int k = (int)(std::upper_bound(rowoff.begin(), rowoff.begin() + nv, dst) - rowoff.begin()) - 1;
    if (dst == rowoff[k] + dep[k]) last[k] = p;
  }
  for (int k = 0; k < nv; ++k)
    if (last[k] >= 0) tasks[4 * last[k] + 3] = (uint32_t)k + 1;
  const int64_t toff = ((5 + (int64_t)levels) + 3) & ~(int64_t)3;
  const int64_t words = toff + (int64_t)tasks.size() + (int64_t)extras.size();
  if (out && capacity >= words) {
    std::fill(out, out + toff, 0u);
    out[0] = (uint32_t)levels;
    out[1] = n_tasks;
    out[2] = (uint32_t)(extras.size() / 2);
    out[3] = (uint32_t)depth_levels;
    std::copy(starts.begin(), starts.end(), out + 4);
    std::copy(tasks.begin(), tasks.end(), out + toff);
    std::copy(extras.begin(), extras.end(), out + toff + tasks.size());
  }
  return words;
}
