"""Operation counts of the propagation kernels, for roofline fractions.

per photon step   7 MUFU  the reference's arithmetic (src/photon_prop_cuda.jl:
                          319-361, 171-241): lg2 for the step length, rcp in
                          the HG formula, sqrt of 1 - cos^2, sin and cos of the
                          azimuth, sqrt(1 - o_z^2) and rsqrt in the rotation (its
                          two divisions by sin(theta) share one rcp), plus the
                          square root of the ray-sphere discriminant when the
                          line meets the sphere; the roofline counts 7.  This
                          kernel issues 7 as well (lg2, sqrt of the
                          discriminant, rcp, sqrt, sin, cos and the turn's
                          rsqrt in physical mode, rcp in the compat-mode
                          rotation), which ncu's opcode counts of the
                          bare-step kernel confirm.
                 ~45 FP32 in the reference's form; this kernel issues 46
                          (ncu: 24 FFMA, 17 FMUL, 5 FADD per step; the
                          physical-mode turn in the meridian frame, without
                          renormalisation).
                  1 Philox2x32-10 block (20 32x32-bit products: half a
                          Philox4x32-10 block, as which it is counted).
per photon start  isotropic: 10 MUFU, 28 FP32; Cherenkov cone: 14 MUFU, 60 FP32;
                  plus one Philox4x32-10 block.
A photon that hits the sphere also re-draws its emission block (rare).
"""

MUFU_PER_STEP_ALG = 7
FP32_PER_STEP_ALG = 45
MUFU_PER_STEP = 7
FP32_PER_STEP = 46
PHILOX_PER_STEP = 0.5  # Philox4x32-10 block equivalents (by 32x32-bit products)
MUFU_PER_PHOTON = {0: 10, 1: 14}   # by emitter type
FP32_PER_PHOTON = {0: 28, 1: 60}
PHILOX_PER_PHOTON = 1


def op_counts(steps, photons_iso, photons_cone, algorithmic=False):
    """(mufu, fp32, Philox4x32-10 block equivalents) for a run; algorithmic=True counts the
    step as the reference's arithmetic does, else as this kernel issues it."""
    m_step = MUFU_PER_STEP_ALG if algorithmic else MUFU_PER_STEP
    f_step = FP32_PER_STEP_ALG if algorithmic else FP32_PER_STEP
    mufu = steps * m_step + photons_iso * MUFU_PER_PHOTON[0] + photons_cone * MUFU_PER_PHOTON[1]
    fp32 = steps * f_step + photons_iso * FP32_PER_PHOTON[0] + photons_cone * FP32_PER_PHOTON[1]
    blocks = steps * PHILOX_PER_STEP + (photons_iso + photons_cone) * PHILOX_PER_PHOTON
    return mufu, fp32, blocks


# ncu figures of the batched kernel as shipped.
# DRAM traffic of one launch of the 4096-pair benchmark batch (5.75e9
# photons), full size, `--metrics dram__bytes_read.sum,dram__bytes_write.sum
# --cache-control none` (one pass): the two timed launches after an L2 flush
# read 2.3 and 3.0 MB and wrote 23.1 and 32.8 MB.  The rest of a step's
# algorithmic bytes (zeroed and accumulated FP64 histograms, hit records)
# stays in the 126 MB L2 during the launch and reaches DRAM afterwards.
NCU_DRAM_BYTES_PER_LAUNCH = 0.5 * ((2.27 + 23.11) + (3.04 + 32.76)) * 1e6
# Issue and pipes on one launch of 512 mixed pairs (<= 1e6 photons each).
NCU_ISSUE_ACTIVE = 0.779
NCU_PIPES = {"alu": 0.518, "fma": 0.395, "xu": 0.375}  # pipe utilisation, same capture
NCU_LANES_ACTIVE = 29.97  # threads per executed warp instruction, same capture
