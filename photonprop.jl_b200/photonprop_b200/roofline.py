"""Operation counts of the propagation kernels, for roofline fractions.

per photon step   7 MUFU  the reference's arithmetic (src/photon_prop_cuda.jl:
                          319-361, 171-241): lg2 for the step length, rcp in
                          the HG formula, sqrt of 1 - cos^2, sin and cos of the
                          azimuth, sqrt(1 - o_z^2) and rsqrt in the rotation (its
                          two divisions by sin(theta) share one rcp), plus the
                          square root of the ray-sphere discriminant when the
                          line meets the sphere; the roofline counts 7.  This
                          kernel issues 7 as well (lg2, sqrt of the
                          discriminant, rcp, sqrt, sin, cos, rcp: the rotation
                          needs no sin(theta) and renormalises with a Newton
                          step), which ncu's opcode counts of the bare-step
                          kernel confirm.
                 ~45 FP32 in the reference's form; this kernel issues 56
                          (ncu: 28 FFMA, 20 FMUL, 8 FADD per step).
                  1 Philox4x32-10 block.
per photon start  isotropic: 10 MUFU, 28 FP32; Cherenkov cone: 14 MUFU, 60 FP32;
                  plus one Philox block.
A photon that hits the sphere also re-draws its emission block (rare).
"""

MUFU_PER_STEP_ALG = 7
FP32_PER_STEP_ALG = 45
MUFU_PER_STEP = 7
FP32_PER_STEP = 56
PHILOX_PER_STEP = 1
MUFU_PER_PHOTON = {0: 10, 1: 14}   # by emitter type
FP32_PER_PHOTON = {0: 28, 1: 60}
PHILOX_PER_PHOTON = 1


def op_counts(steps, photons_iso, photons_cone, algorithmic=False):
    """(mufu, fp32, philox blocks) for a run; algorithmic=True counts the
    step as the reference's arithmetic does, else as this kernel issues it."""
    m_step = MUFU_PER_STEP_ALG if algorithmic else MUFU_PER_STEP
    f_step = FP32_PER_STEP_ALG if algorithmic else FP32_PER_STEP
    mufu = steps * m_step + photons_iso * MUFU_PER_PHOTON[0] + photons_cone * MUFU_PER_PHOTON[1]
    fp32 = steps * f_step + photons_iso * FP32_PER_PHOTON[0] + photons_cone * FP32_PER_PHOTON[1]
    blocks = steps * PHILOX_PER_STEP + (photons_iso + photons_cone) * PHILOX_PER_PHOTON
    return mufu, fp32, blocks


# DRAM traffic of the batched kernel per photon, measured with ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) on one launch of 2.524e8
# photons (512 mixed pairs, <= 1e6 photons each): 117.8 KB read, 0 B written.
# Hit records and FP64 histogram reductions stay in L2 during a launch, so
# the traffic grows with the photon count; bench.py scales it to its launch.
NCU_DRAM_BYTES_PER_PHOTON = 117.76e3 / 252387747
# Issue slots busy in the same capture (smsp__issue_active).
NCU_ISSUE_ACTIVE = 0.775
NCU_PIPES = {"alu": 0.503, "fma": 0.338, "xu": 0.284}  # pipe utilisation, same capture
NCU_BRANCH_UNIFORM = 0.914  # smsp__sass_average_branch_targets_threads_uniform, same capture
