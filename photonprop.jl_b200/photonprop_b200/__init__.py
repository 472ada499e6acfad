"""photonprop_b200: B200-native photon propagation for PhotonProp.jl.

Python host mirror of the reference's Julia API (Medium, Spectral, Emission,
Detection and PhotonPropagationCuda modules) over the C ABI of
libphotonprop_b200.so, whose CUDA kernels (sm_100a) do all propagation.
"""
from . import _lib
from ._lib import EXPORTED, HIT_DTYPE, PAIR_DTYPE, PPError
from .detection import DetectionSphere, PMTWavelengthAcceptance, p_one_pmt_acc, p_one_pmt_acc_5nm
from .emission import (AngularEmissionProfile, CherenkovEmission, IsotropicEmission, PhotonSource,
                       cherenkov_ang_dist)
from .medium import (WaterProperties, get_absorption_length, get_group_index, get_refractive_index,
                     get_scattering_length, make_cascadia_medium_properties, make_seawater)
from .propagation import (PropagationResult, Propagator, RunOptions, cuda_propagate_photons_,
                          initialize_photon_arrays, make_pair, pair_seed, process_output,
                          propagate_distance)
from .spectrum import CherenkovSpectrum, Monochromatic, Spectrum
from . import batches
from . import serving
from . import parallel
from . import surrogate
from . import modelling
from . import lightyield
from . import event


def build(force=False):
    from . import _build
    return _build.build(force=force)


def launch_count() -> int:
    return int(_lib.load().pp_launch_count())


def measure_peaks(device=0):
    """FP32 FMA and MUFU issue peaks (ops/s) and the Philox4x32-10 block rate
    (blocks/s) of the device."""
    import ctypes
    L = _lib.load()
    f, m, i = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    _lib.check(L.pp_measure_peaks(device, ctypes.byref(f), ctypes.byref(m), ctypes.byref(i)))
    return {"fp32_ops": f.value, "mufu_ops": m.value, "philox_blocks": i.value}


def measure_step_rate(device=0):
    """Photon steps per second of the bare physical step on every SM (one
    Philox2x32 block, ray-sphere test, move, turn; no emission, refill, hit
    record or loop bookkeeping): the speed of light of the step loop."""
    import ctypes
    L = _lib.load()
    r = ctypes.c_double()
    _lib.check(L.pp_measure_step_rate(device, ctypes.byref(r)))
    return r.value
