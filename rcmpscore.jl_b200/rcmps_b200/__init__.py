"""B200-native fg_phi4: the phi^4 energy density and gradient of relativistic continuous matrix
product states, on sm_100a kernels behind the C ABI of include/rcmps_b200.h.

The host API mirrors rcmps_gpu (RcmpsCore.jl's GPU package): the portable state format
(rcmps_b200.io), the objective callable and its components (rcmps_b200.objective).
"""
__version__ = "0.1.0"
