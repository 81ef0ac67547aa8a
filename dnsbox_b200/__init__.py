"""dnsbox_b200: B200-native pseudospectral Navier-Stokes time step of dnsbox.

The compute path is the C-ABI library ``libdnsbox_gpu.so`` (hand-written
sm_100a CUDA kernels, see ``csrc/``); ``ops`` binds it for PyTorch tensors.
Importing the package does not load the library; the first call into ``ops``
does, and raises if the library or a GPU is missing (there is no CPU path).
"""
__all__ = ["grid", "ic"]
