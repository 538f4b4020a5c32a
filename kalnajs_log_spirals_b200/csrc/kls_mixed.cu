// Split-BF16 tensor-core contraction (KLS_MODE_MIXED).
#include "kls_internal.cuh"

struct kls_mixed {};

int kls_mixed_prepare(kls_ctx* c) {
  return kls_fail(c, KLS_ERR_UNSUPPORTED, "mixed-precision contraction not built yet");
}

int kls_mixed_contract(kls_ctx* c, int, int) {
  return kls_fail(c, KLS_ERR_UNSUPPORTED, "mixed-precision contraction not built yet");
}

void kls_mixed_free(kls_ctx* c) {
  delete c->mixed;
  c->mixed = nullptr;
}
