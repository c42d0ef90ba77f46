// fast.cu -- fused fast path (CONFIG mode); filled in below the canonical path.
#include "state.cuh"
namespace symb200 {
int fast_alloc(sym_handle* h) { h->fast.storage = -1; return SYM_OK; }
void fast_free(sym_handle* h) { (void)h; }
int fast_import(sym_handle* h) { return set_error(h, SYM_ERR_UNSUPPORTED, "fast path not built"); }
int fast_export(sym_handle* h) { return set_error(h, SYM_ERR_UNSUPPORTED, "fast path not built"); }
int fast_step(sym_handle* h, int n) { (void)n; return set_error(h, SYM_ERR_UNSUPPORTED, "fast path not built"); }
}  // namespace symb200
