// merge.cu — the table of kernels that have a merged form (merge.cuh), filled as the library loads.
#include <unordered_map>

#include "merge.cuh"

namespace tdgl {

static std::unordered_map<const void *, MergeInfo> &merge_table() {
  static std::unordered_map<const void *, MergeInfo> t;
  return t;
}

void merge_register(const void *kern, MergeInfo m) { merge_table()[kern] = m; }

const MergeInfo *merge_lookup(const void *kern) {
  auto &t = merge_table();
  auto it = t.find(kern);
  return it == t.end() ? nullptr : &it->second;
}

}  // namespace tdgl
