"""frfs_b200: a B200-native (sm_100a) implementation of the DGFS hot path
of jaisw7/frfs -- the fast-spectral Boltzmann collision operator and the
flux-reconstruction advection operators -- behind the reference's
.ini-driven system, kernel-name and integrator interface.
"""
__version__ = '0.1.0'
