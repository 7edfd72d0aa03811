// A reference-side Surface that builds its SES patches with libnsgpu's host builder and ray casts
// on the GPU: the C++ binding INTEGRATION.md describes, compiled by the test suite against a
// stand-in of the reference's interface (reference_stub/Surface.h).
#pragma once
#include <cstdint>
#include <set>
#include <vector>

#include "Surface.h"
#include "nsgpu.h"

class GpuSesSurface : public Surface {
 public:
  explicit GpuSesSurface(DelPhiShared* ds, double probe = 1.4, int precision = NSG_PRECISION_FP64)
      : probe_radius(probe), precision_(precision) {
    delphi = ds;
  }
  ~GpuSesSurface() override {
    if (ctx) nsg_ctx_destroy(ctx);
    if (patches) nsg_patchset_free(patches);
  }

  // ConnollySurface::build: the SES patches of the (jittered) atoms, on the host.
  bool build() override {
    std::vector<double> xyzr(4 * delphi->atoms.size());
    for (size_t i = 0; i < delphi->atoms.size(); i++) {
      for (int d = 0; d < 3; d++) xyzr[4 * i + d] = delphi->atoms[i].pos[d];
      xyzr[4 * i + 3] = delphi->atoms[i].radius;
    }
    int64_t seed = 1234;
    if (nsg_jitter_atoms(xyzr.data(), (int64_t)delphi->atoms.size(), 1e-4, &seed) != NSG_OK) return false;
    // the reference jitters DelPhiShared's atoms in place; cavity atoms use them
    for (size_t i = 0; i < delphi->atoms.size(); i++)
      for (int d = 0; d < 3; d++) delphi->atoms[i].pos[d] = xyzr[4 * i + d];
    atoms_xyzr = xyzr;
    if (patches) nsg_patchset_free(patches);
    patches = nullptr;
    return nsg_ses_build(xyzr.data(), (int64_t)delphi->atoms.size(), probe_radius, 0, &patches) == NSG_OK;
  }

  bool getSurf(double* surf_vol, bool, bool fill, double cav_vol, vector<packet>*) override {
    if (!patches) return false;
    if (!ctx && nsg_ctx_create(0, &ctx) != NSG_OK) return false;
    NsGrid g{};
    g.nx = delphi->nx; g.ny = delphi->ny; g.nz = delphi->nz;
    g.xmin = delphi->xmin; g.ymin = delphi->ymin; g.zmin = delphi->zmin;
    g.xmax = delphi->xmax; g.ymax = delphi->ymax; g.zmax = delphi->zmax;
    g.scale = delphi->scale; g.side = delphi->side; g.hside = delphi->hside; g.A = delphi->A;
    g.rmaxdim = delphi->rmaxdim;
    for (int d = 0; d < 3; d++) g.baricenter[d] = delphi->baricenter[d];
    int64_t n = 0, npool = 0, counts[5];
    if (nsg_patchset_info(patches, &n, &npool, counts) != NSG_OK) return false;
    std::vector<double> f64(20 * n), pool(4 * (npool > 0 ? npool : 1));
    std::vector<int32_t> i32(4 * n);
    std::vector<int8_t> flag(npool > 0 ? npool : 1);
    if (nsg_patchset_export(patches, f64.data(), i32.data(), pool.data(), flag.data()) != NSG_OK) return false;
    if (nsg_set_grid(ctx, &g) != NSG_OK ||
        nsg_upload_patches(ctx, n, f64.data(), i32.data(), npool, pool.data(), flag.data(), probe_radius) != NSG_OK)
      return false;
    const int flags = (delphi->buildStatus ? NSG_RAYCAST_STATUS : 0) | (accurateTriangulation ? NSG_RAYCAST_TRIANGULATION : 0);
    if (nsg_raycast(ctx, flags, precision_, surf_vol) != NSG_OK) return false;
    if (fill) {
      int ncav = 0;
      if (nsg_cavities(ctx, cav_vol, &ncav) != NSG_OK) return false;
      delphi->cavitiesSize.assign(ncav, 0.0);
      std::vector<int32_t> filled(ncav);
      if (ncav > 0 && nsg_download_cavities(ctx, delphi->cavitiesSize.data(), filled.data()) != NSG_OK) return false;
      delphi->cavitiesFlag.assign(filled.begin(), filled.end());
      // getCavitiesAtomsWithBilevelStatusMap: cav2atoms, one set per cavity
      int64_t total = 0;
      const int64_t na = (int64_t)atoms_xyzr.size() / 4;
      if (nsg_cavity_atoms(ctx, atoms_xyzr.data(), na, nullptr, nullptr, &total) != NSG_OK) return false;
      std::vector<int32_t> off(ncav + 1), lst(total > 0 ? total : 1);
      if (nsg_cavity_atoms(ctx, atoms_xyzr.data(), na, off.data(), lst.data(), &total) != NSG_OK) return false;
      for (auto* st : delphi->cav2atoms) delete st;
      delphi->cav2atoms.assign(ncav, nullptr);
      for (int cv = 0; cv < ncav; cv++) delphi->cav2atoms[cv] = new std::set<int>(&lst[off[cv]], &lst[off[cv + 1]]);
    }
    if (delphi->buildStatus && delphi->status && nsg_download_status(ctx, delphi->status) != NSG_OK) return false;
    return true;
  }

  double triangulateSurface(bool, bool, double, const char*, bool) override {
    double area = 0;
    int64_t nv = 0, nt = 0;
    if (!ctx || nsg_triangulate(ctx, &area, &nv, &nt) != NSG_OK) return -1;
    vertList.assign(3 * nv, 0.0);
    triList.assign(3 * nt, 0);
    std::vector<int32_t> keys(4 * nv);
    if (nsg_download_mesh(ctx, vertList.data(), keys.data(), triList.data()) != NSG_OK) return -1;
    return area;
  }

 private:
  nsg_ctx* ctx = nullptr;
  NsPatchSet* patches = nullptr;
  std::vector<double> atoms_xyzr;  // the jittered atoms (x, y, z, r)
  double probe_radius;
  int precision_;
};
