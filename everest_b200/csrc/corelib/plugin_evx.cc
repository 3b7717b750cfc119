// The worker plugin: exports the reference's factory symbol
// `extern "C" GPUWorker *getWorker(int gpu)`
// (system/templates/GPUWorker/interface.snp:1-7).  One prebuilt plugin serves
// every motif; the motif arrives with the job at take() time.
#include <stdexcept>

#include "corelib.h"

extern "C" __attribute__((visibility("default"))) corelib::GPUWorker *getWorker(int gpu) {
  try {
    return new corelib::GPUWorkerEVX(gpu);
  } catch (const std::exception &) {
    return nullptr;  // the loader reports evx_last_error()
  }
}
