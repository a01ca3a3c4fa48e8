// Plain-form (FP64) instantiations of the primitive-variable sweep and the precision dispatch.
// The kernels and Riemann solvers live in inviscid_pv.cuh; the FP32 (mixed-form) instantiations
// are compiled in inviscid_pv_f32.cu.
#include "inviscid_pv.cuh"

namespace cb2 {

template <int NS, int SOLVER, bool TT = false>
static int launch_pv_rec(const Zone &z, const Param &p, cudaStream_t s, int &nl) {
  switch (p.reconstruction) {
    case CB2_REC_MUSCL: return launch_pv_dirs<double, NS, 2, SOLVER, TT>(z, p, s, nl);
    case CB2_REC_NND2: return launch_pv_dirs<double, NS, 3, SOLVER, TT>(z, p, s, nl);
    case CB2_REC_WENO5: return launch_pv_dirs<double, NS, 5, SOLVER, TT>(z, p, s, nl);
    case CB2_REC_WENO7: return launch_pv_dirs<double, NS, 7, SOLVER, TT>(z, p, s, nl);
    default: return launch_pv_dirs<double, NS, 1, SOLVER, TT>(z, p, s, nl);
  }
}

// Two temperatures (FP64): AUSM+ and HLLC over the n_spec species and e_ve (NSC = n_spec + 1
// scalars); the reference's two-temperature build has no Roe or Lax-Friedrichs variant.
template <int NSC>
static int launch_pv_2t(const Zone &z, const Param &p, cudaStream_t s, int &nl) {
  switch (p.inviscid_scheme) {
    case CB2_INV_AUSMP: return launch_pv_rec<NSC, CB2_INV_AUSMP, true>(z, p, s, nl);
    case CB2_INV_HLLC: return launch_pv_rec<NSC, CB2_INV_HLLC, true>(z, p, s, nl);
    default: return CB2_ERR_UNSUPPORTED;
  }
}

template <int NS>
static int launch_pv_ns(const Zone &z, const Param &p, cudaStream_t s, int &nl) {
  switch (p.inviscid_scheme) {
    case CB2_INV_AUSMP: return launch_pv_rec<NS, CB2_INV_AUSMP>(z, p, s, nl);
    case CB2_INV_HLLC: return launch_pv_rec<NS, CB2_INV_HLLC>(z, p, s, nl);
    case CB2_INV_ROE: return launch_pv_rec<NS, CB2_INV_ROE>(z, p, s, nl);
    case 1:
      if constexpr (NS == 0) return launch_pv_rec<0, 1>(z, p, s, nl);
      else return CB2_ERR_UNSUPPORTED;
    default: return CB2_ERR_UNSUPPORTED;
  }
}

int launch_inviscid_pv(const Zone &z, const Param &p, cudaStream_t s, int &n_launch) {
  if (p.precision == CB2_PREC_MIXED) return launch_inviscid_pv_f32(z, p, s, n_launch);
  if (p.i_eve >= 0) {
    switch (p.n_spec) {
      case 5: return launch_pv_2t<6>(z, p, s, n_launch);
      case 9: return launch_pv_2t<10>(z, p, s, n_launch);
      default: return CB2_ERR_UNSUPPORTED;
    }
  }
  switch (p.n_spec) {
    case 0: return launch_pv_ns<0>(z, p, s, n_launch);
    case 5: return launch_pv_ns<5>(z, p, s, n_launch);
    case 9: return launch_pv_ns<9>(z, p, s, n_launch);
    default: return CB2_ERR_UNSUPPORTED;
  }
}

}  // namespace cb2
