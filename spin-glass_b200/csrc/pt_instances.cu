// pt_instances.cu — the resident kernel's instantiations for one lattice side.
// The build compiles this file once per L with -DCSG_PT_L=<L> (the
// instantiations of different L compile in parallel); the host code finds them
// through resident_kernel_L<L>() (pt_kernel.cuh).
#include "pt_resident.cuh"

#ifndef CSG_PT_L
#error "build with -DCSG_PT_L=<lattice side>"
#endif

namespace csg {
namespace {

template <int L, int I>
ResidentFn pick(bool gen, int nseg) {
    constexpr int NS = nseg_option(L, I);
    if constexpr (NS > 0) {
        if (nseg == NS) return gen ? pt_resident_kernel<L, true, NS> : pt_resident_kernel<L, false, NS>;
        return pick<L, I + 1>(gen, nseg);
    } else {
        return nullptr;
    }
}

}  // namespace

#define CSG_CAT2(a, b) a##b
#define CSG_CAT(a, b) CSG_CAT2(a, b)
ResidentFn CSG_CAT(resident_kernel_L, CSG_PT_L)(bool gen, int nseg) { return pick<CSG_PT_L, 0>(gen, nseg); }

}  // namespace csg
