// Minimal stand-in for the reference's plugin interface, declaring only the members that
// tests/cxx/gpu_ses_surface.h uses, with the reference's names and signatures
// (src/Surface.h:835-990, src/DelphiShared.h:151-213, src/nanoshaper.h:227-292).  It exists so that
// the GPU Surface subclass shown in INTEGRATION.md compiles in the test suite; it is not the
// reference's header.
#pragma once
#include <cstdint>
#include <set>
#include <string>
#include <vector>

using std::vector;

class Atom {
 public:
  double pos[3];
  double radius;
};

class DelPhiShared {
 public:
  int64_t nx, ny, nz;
  double xmin, xmax, ymin, ymax, zmin, zmax;
  double scale, side, hside, A, rmaxdim;
  double baricenter[3];
  bool buildStatus;
  int* status;
  std::vector<Atom> atoms;
  vector<double> cavitiesSize;
  vector<bool> cavitiesFlag;
  vector<std::set<int>*> cav2atoms;
  ~DelPhiShared() {
    for (auto* s : cav2atoms) delete s;
  }
};

struct packet;

class Surface {
 public:
  virtual ~Surface() {}
  virtual bool build(void) = 0;
  virtual bool getSurf(double* surf_vol, bool optimize_grids, bool fill = false, double cav_vol = 0,
                       vector<packet>* intersectionsInfo = nullptr) = 0;
  virtual double triangulateSurface(bool outputMesh, bool buildAtomsMapHere, double iso = 0.0,
                                    const char* fileName = "triangulatedSurf", bool revert = false) = 0;

 protected:
  DelPhiShared* delphi = nullptr;
  bool accurateTriangulation = true;
  vector<int> triList;
  vector<double> vertList;
};
