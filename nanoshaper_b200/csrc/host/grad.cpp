// Chain rule from per-patch surface parameters to atom coordinates and radii (host); the
// per-patch math is chain_patch (chain.h), which the device chain kernel shares.
#include <cstring>

#include "../chain.h"
#include "host_api.h"

extern "C" {

// grad_atoms (n_atoms x 4: x, y, z, r) += d out / d atoms, from the per-patch parameter gradients
// gpatch (n_patches x NS_GRAD_PER_PATCH).  atoms_xyzr are the atoms the patches were built from
// (after any jitter); patch_atoms holds 3 atom indices per patch (nsg_patchset_atoms).
int nsg_ses_chain_grad(const double* atoms_xyzr, int64_t n_atoms, double probe, int64_t n_patches,
                       const int32_t* i32, const double* f64, const int32_t* patch_atoms, const double* gpatch,
                       double* grad_atoms) {
  if (!atoms_xyzr || !i32 || !f64 || !patch_atoms || !gpatch || !grad_atoms || n_atoms < 0 || n_patches < 0)
    return NSG_ERR_ARG;
  int n_bad = 0;
  auto add = [grad_atoms](int32_t atom, int slot, double v) { grad_atoms[4 * atom + slot] += v; };
  for (int64_t p = 0; p < n_patches; p++) {
    const int32_t* pa = patch_atoms + 3 * p;
    for (int q = 0; q < 3; q++)
      if (pa[q] >= n_atoms) return NSG_ERR_ARG;
    if (!nsg::chain_patch(i32[NS_PATCH_I32 * p], f64 + NS_PATCH_F64 * p, pa, atoms_xyzr, probe,
                          gpatch + NS_GRAD_PER_PATCH * p, add))
      n_bad++;
  }
  return n_bad ? NSG_ERR_GEOMETRY : NSG_OK;
}

}  // extern "C"
