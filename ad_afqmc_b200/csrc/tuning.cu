// Process-wide registry of tile/schedule records (afq_tuning), keyed by the
// layout-relevant fields of afq_dims.  make_layout() consults it on every call.
#include <map>
#include <mutex>
#include <tuple>

#include "layout.cuh"

namespace afq {
namespace {

using Key = std::tuple<int, int, int, int, int, int, int, int>;

Key key_of(const afq_dims& d) {
  const int nb = d.walker_type == AFQ_RESTRICTED ? d.nocc[0] : d.nocc[1];
  return Key(d.norb, d.nocc[0], nb, d.nchol, d.nwalkers, d.walker_type, d.trial_type, d.precision);
}

std::mutex& registry_mutex() {
  static std::mutex m;
  return m;
}

std::map<Key, afq_tuning>& registry() {
  static std::map<Key, afq_tuning> r;
  return r;
}

}  // namespace

bool tuning_lookup(const afq_dims& d, afq_tuning& out) {
  std::lock_guard<std::mutex> g(registry_mutex());
  auto& r = registry();
  if (r.empty()) return false;
  auto it = r.find(key_of(d));
  if (it == r.end()) return false;
  out = it->second;
  return true;
}

void tuning_store(const afq_dims& d, const afq_tuning* t) {
  std::lock_guard<std::mutex> g(registry_mutex());
  if (t)
    registry()[key_of(d)] = *t;
  else
    registry().erase(key_of(d));
}

}  // namespace afq
