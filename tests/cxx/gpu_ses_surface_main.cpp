// Links the GPU Surface subclass against libnsgpu.so (compile and link check; it runs only when a
// GPU is present).
#include <cstdio>

#include "gpu_ses_surface.h"

int main() {
  DelPhiShared ds{};
  ds.buildStatus = true;
  GpuSesSurface s(&ds);
  std::printf("GpuSesSurface %p\n", (void*)&s);
  return 0;
}
