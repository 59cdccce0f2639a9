/* Build configuration for the oracle's CPU-only build of the reference fitter
 * (the reference generates this header from config.hh.in with CMake). */
#define Tempest_VERSION_MAJOR 0
#define Tempest_VERSION_MINOR 1
#define HAS_SSE
#define DISABLE_CUDA
