// k_learned.cu — learned preconditioner (placeholder until its kernels land).
#include "llg_internal.h"

struct Learned {
  int unused;
};

void learned_destroy(Learned* l) { delete l; }
