// Host-owned patch set: the output of the patch builders (SES, skin) in the layout the ray caster
// uploads (see ns_types.h and include/nsgpu.h).
#pragma once
#include <stdint.h>

#include <vector>

#include "../ns_types.h"

struct NsPatchSet {
  std::vector<double> f64;
  std::vector<int32_t> i32;
  std::vector<double> pool;
  std::vector<int8_t> pool_flag;
  std::vector<int32_t> atoms;  // 3 per patch: the atoms the patch's surface depends on, -1 unused
  int64_t counts[NS_KIND_COUNT] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  void add_patch(int kind, const double* rec, const double* pool4, const int8_t* flags, int64_t npool, int32_t a0,
                 int32_t a1, int32_t a2) {
    atoms.push_back(a0);
    atoms.push_back(a1);
    atoms.push_back(a2);
    int64_t first = (int64_t)pool_flag.size();
    f64.insert(f64.end(), rec, rec + NS_PATCH_F64);
    i32.push_back(kind);
    i32.push_back((int32_t)first);
    i32.push_back((int32_t)npool);
    i32.push_back(0);
    if (npool) {
      pool.insert(pool.end(), pool4, pool4 + 4 * npool);
      if (flags) pool_flag.insert(pool_flag.end(), flags, flags + npool);
      else pool_flag.insert(pool_flag.end(), (size_t)npool, (int8_t)0);
    }
    counts[kind]++;
  }
};

