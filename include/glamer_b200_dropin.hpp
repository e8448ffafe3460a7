// Settings of the link-level drop-in (slsimlib_b200/dropin/glamer_b200_dropin.cpp),
// which defines GLAMER's Lens::rayshooter / Lens::rayshooterInternal on the
// GPU.  Include after GLAMER's lens.h.
#ifndef GLAMER_B200_DROPIN_HPP
#define GLAMER_B200_DROPIN_HPP

class Lens;

namespace glamer_b200_dropin {

// Precision of the tree walk for every lens shot through the drop-in:
// GLB_PREC_FP64 (default, the reference's arithmetic) or GLB_PREC_SPLIT.
void set_precision(int precision);

// Frees the device mirror of `lens` (call before the Lens is destroyed when
// the process keeps running; mirrors otherwise live until exit).
void release(const Lens *lens);

}  // namespace glamer_b200_dropin

#endif
