// Internal view of a built hf_ctx for the other translation units.
#pragma once
#include <stdint.h>

#include "hfjk.h"

namespace hf {

struct TensorView {
    int device;
    const double* B;  // [naux][ntiles][64][64]
    int64_t n;
    int nt;
    int64_t ntiles;
    int naux;
    bool built;
};

// Fills *out from ctx; HF_ERR_ARG for a null context.
int context_view(const hf_ctx* ctx, TensorView* out);

}  // namespace hf
