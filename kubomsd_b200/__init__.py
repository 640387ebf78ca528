"""B200-native stochastic-KPM transport backend for KuboMSD.

The hot path (Chebyshev/KPM moments, Bessel propagation with the velocity
commutator, batched PCG metric solves, metric sampling) runs in
libkmsd_b200.so, hand-written CUDA for sm_100a behind a C ABI
(include/kmsd.h).  This package holds the host side: the reference-facing
adapter (`native`), the operator bundle (`operators`), the device-resident
stochastic driver (`stochastic`), host formulas (`kpm`), model/result I/O
(`io`), the CLI (`cli`) and the synthetic workloads (`lattices`).
"""
__version__ = "0.1.0"
