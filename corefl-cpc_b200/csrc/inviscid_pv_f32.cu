// Mixed-form (FP32 arithmetic) instantiations of the primitive-variable sweep: WENO5/WENO7
// reconstruction with the AUSM+, HLLC and Roe fluxes.  The field arrays stay FP64; node data
// is rounded to FP32 as it is staged into shared memory and the FP32 flux difference is added
// to the FP64 dq.
#include "inviscid_pv.cuh"

namespace cb2 {

template <int NS, int SOLVER>
static int launch_pv32_rec(const Zone &z, const Param &p, cudaStream_t s, int &nl) {
  switch (p.reconstruction) {
    case CB2_REC_WENO5: return launch_pv_dirs<float, NS, 5, SOLVER>(z, p, s, nl);
    case CB2_REC_WENO7: return launch_pv_dirs<float, NS, 7, SOLVER>(z, p, s, nl);
    default: return CB2_ERR_UNSUPPORTED;
  }
}

template <int NS>
static int launch_pv32_ns(const Zone &z, const Param &p, cudaStream_t s, int &nl) {
  switch (p.inviscid_scheme) {
    case CB2_INV_AUSMP: return launch_pv32_rec<NS, CB2_INV_AUSMP>(z, p, s, nl);
    case CB2_INV_HLLC: return launch_pv32_rec<NS, CB2_INV_HLLC>(z, p, s, nl);
    case CB2_INV_ROE: return launch_pv32_rec<NS, CB2_INV_ROE>(z, p, s, nl);
    default: return CB2_ERR_UNSUPPORTED;
  }
}

int launch_inviscid_pv_f32(const Zone &z, const Param &p, cudaStream_t s, int &n_launch) {
  switch (p.n_spec) {
    case 0: return launch_pv32_ns<0>(z, p, s, n_launch);
    case 5: return launch_pv32_ns<5>(z, p, s, n_launch);
    case 9: return launch_pv32_ns<9>(z, p, s, n_launch);
    default: return CB2_ERR_UNSUPPORTED;
  }
}

}  // namespace cb2
