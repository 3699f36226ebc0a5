// Internal definition of the H_eff operator object (shared by heff.cu and the
// Lanczos solver).
#pragma once

#include "blocksparse.h"
#include "gemm.cuh"

namespace dmrg {
struct LanczosWork;
}

struct dmrg_heff_s {
    dmrg_ctx_t ctx = nullptr;
    int precision = DMRG_PREC_FP64;
    int64_t split_min_dim = 200000;  // psi_dim from which a split operator's Lanczos starts with a split phase
    bool use_graph = true;            // Lanczos loop as one captured CUDA graph (dmrg_heff_set_graph)
    dmrg::SiteDesc site;
    dmrg::EnvDesc L, R;
    dmrg::GemmSchedule sa, sb;    // A: psi x R -> T ; B: L x T -> out (FP64 tiles)
    // split precisions (DMRG_PREC_TF32X3 / DMRG_PREC_BF16X3) only: operand images
    // and packed schedules
    dmrg::PackSchedule pk_psi, pk_L, pk_R;     // which blocks to pack, where
    dmrg::PackedSchedule pa, pb;               // A: psi x R -> T images ; B: L x T -> out
    dmrg::DeviceBuffer img_psi, img_L, img_R, img_T;
    int64_t t_img_bytes = 0;
    dmrg::DeviceBuffer T;
    int64_t t_size = 0;
    const double* L_dev = nullptr;
    const double* R_dev = nullptr;
    double flops_alg = 0, flops_exec = 0;
    dmrg::DeviceBuffer io_psi, io_out;  // staging for dmrg_heff_apply_host
    dmrg::LanczosWork* lw = nullptr;  // Lanczos workspace, allocated on first use
    ~dmrg_heff_s();
};

namespace dmrg {
inline bool is_split(int precision) { return precision == DMRG_PREC_TF32X3 || precision == DMRG_PREC_BF16X3; }
inline int split_fmt(int precision) { return precision == DMRG_PREC_BF16X3 ? kFmtBF16 : kFmtTF32; }
// out (+)= H_eff psi on the context stream, in the operator's precision.
int heff_apply_internal(dmrg_heff_s& h, const double* psi, double* out, bool accumulate);
// out (+)= H_eff psi in FP64 whatever the operator's precision.
int heff_apply_fp64(dmrg_heff_s& h, const double* psi, double* out, bool accumulate);
}  // namespace dmrg
