// Mixed-size submission of single-map transforms (ps_batch_submit): the items are
// grouped by (plan, direction, spin, scale) and each group runs as one batched
// transform, largest groups (pixels x maps) first.  Inputs and outputs that already
// lie back to back in item order are used in place; others go through staging
// buffers in the workspace with one device-to-device copy per item.  All launches
// and copies are asynchronous on one stream, so a submission is capturable.
#include <algorithm>
#include <map>
#include <tuple>
#include <vector>

#include "ps_common.cuh"

namespace {

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

struct Group {
  const ps_plan* plan;
  int dir, spin;
  double scale;
  std::vector<int> items;
  size_t in_bytes, out_bytes;  // per map
  int64_t weight;              // pixels x maps, for the order
  bool in_contig, out_contig;
  size_t ws_sht;
};

int make_groups(const ps_work_item* items, int n, std::vector<Group>& groups) {
  std::map<std::tuple<const ps_plan*, int, int, double>, int> index;
  for (int i = 0; i < n; ++i) {
    const ps_work_item& it = items[i];
    if (!it.plan || (it.direction != PS_DIR_SYNTHESIS && it.direction != PS_DIR_ADJOINT) || it.spin < 0 ||
        it.spin > 3 || !it.in || !it.out)
      return PS_ERR_INVALID;
    const double sc = it.direction == PS_DIR_ADJOINT ? it.scale : 0.0;
    const auto key = std::make_tuple(it.plan, it.direction, it.spin, sc);
    auto f = index.find(key);
    if (f == index.end()) {
      int64_t npix = 0, nalm = 0;
      const int rc = ps_plan_info(it.plan, nullptr, nullptr, &npix, &nalm);
      if (rc != PS_OK) return rc;
      const size_t nc = it.spin == 0 ? 1 : 2;
      Group g;
      g.plan = it.plan;
      g.dir = it.direction;
      g.spin = it.spin;
      g.scale = sc;
      const size_t alm_b = nc * size_t(nalm) * sizeof(double2), map_b = nc * size_t(npix) * sizeof(double);
      g.in_bytes = it.direction == PS_DIR_SYNTHESIS ? alm_b : map_b;
      g.out_bytes = it.direction == PS_DIR_SYNTHESIS ? map_b : alm_b;
      g.weight = npix;
      f = index.emplace(key, int(groups.size())).first;
      groups.push_back(g);
    }
    groups[size_t(f->second)].items.push_back(i);
  }
  for (Group& g : groups) {
    g.weight *= int64_t(g.items.size());
    g.in_contig = g.out_contig = true;
    for (size_t k = 1; k < g.items.size(); ++k) {
      const ps_work_item& a = items[g.items[k - 1]];
      const ps_work_item& b = items[g.items[k]];
      if (reinterpret_cast<const char*>(b.in) != reinterpret_cast<const char*>(a.in) + g.in_bytes) g.in_contig = false;
      if (reinterpret_cast<const char*>(b.out) != reinterpret_cast<const char*>(a.out) + g.out_bytes)
        g.out_contig = false;
    }
    const int rc = ps_sht_workspace_bytes(g.plan, int(g.items.size()), g.spin, g.dir, &g.ws_sht);
    if (rc != PS_OK) return rc;
  }
  std::stable_sort(groups.begin(), groups.end(), [](const Group& a, const Group& b) { return a.weight > b.weight; });
  return PS_OK;
}

size_t group_bytes(const Group& g) {
  const size_t B = g.items.size();
  return (g.in_contig ? 0 : al256(B * g.in_bytes)) + (g.out_contig ? 0 : al256(B * g.out_bytes)) +
         al256(std::max<size_t>(g.ws_sht, 256));
}

}  // namespace

extern "C" int ps_batch_workspace_bytes(const ps_work_item* items, int n, size_t* bytes) {
  if (!bytes || n < 0 || (n > 0 && !items)) return PS_ERR_INVALID;
  std::vector<Group> groups;
  const int rc = make_groups(items, n, groups);
  if (rc != PS_OK) return rc;
  size_t need = 256;
  for (const Group& g : groups) need = std::max(need, group_bytes(g));
  *bytes = need;
  return PS_OK;
}

extern "C" int ps_batch_submit(const ps_work_item* items, int n, void* workspace, size_t workspace_bytes,
                               cudaStream_t stream) {
  if (n < 0 || (n > 0 && !items)) return PS_ERR_INVALID;
  if (n == 0) return PS_OK;
  std::vector<Group> groups;
  int rc = make_groups(items, n, groups);
  if (rc != PS_OK) return rc;
  size_t need = 256;
  for (const Group& g : groups) need = std::max(need, group_bytes(g));
  if (!workspace || workspace_bytes < need) return PS_ERR_WORKSPACE;
  char* ws = static_cast<char*>(workspace);
  for (const Group& g : groups) {
    const int B = int(g.items.size());
    char* p = ws;
    const double* in = items[g.items[0]].in;
    double* out = items[g.items[0]].out;
    if (!g.in_contig) {
      for (int k = 0; k < B; ++k)
        if (cudaMemcpyAsync(p + size_t(k) * g.in_bytes, items[g.items[size_t(k)]].in, g.in_bytes,
                            cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
          return PS_ERR_CUDA;
      in = reinterpret_cast<const double*>(p);
      p += al256(size_t(B) * g.in_bytes);
    }
    if (!g.out_contig) {
      out = reinterpret_cast<double*>(p);
      p += al256(size_t(B) * g.out_bytes);
    }
    const size_t ws_left = workspace_bytes - size_t(p - ws);
    rc = g.dir == PS_DIR_SYNTHESIS ? ps_synthesis(g.plan, in, out, B, g.spin, p, ws_left, stream)
                                   : ps_adjoint(g.plan, in, out, B, g.spin, g.scale, p, ws_left, stream);
    if (rc != PS_OK) return rc;
    if (!g.out_contig)
      for (int k = 0; k < B; ++k)
        if (cudaMemcpyAsync(items[g.items[size_t(k)]].out, reinterpret_cast<const char*>(out) + size_t(k) * g.out_bytes,
                            g.out_bytes, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
          return PS_ERR_CUDA;
  }
  return PS_OK;
}
