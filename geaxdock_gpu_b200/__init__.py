"""B200-native replica-exchange Monte Carlo docking engine (GeauxDock's MonteCarlo_d path).

The compute path is the CUDA library geaxdock_gpu_b200/libgeauxdock_b200.so behind the C ABI
declared in include/geauxdock_b200.h; this package holds its ctypes mirror (abi), the
host-side mirror of the reference's Run/MonteCarlo_d interface (engine) and the synthetic
workload generator (system).
"""
__all__ = ["abi"]
