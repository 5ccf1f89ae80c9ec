"""B200-native drop-in for the curved-boundary vectorial LBM solvers.

Same package layout as the reference ``curved_lbm`` (1.0.0): ``two_d`` holds
the D2Q4x6 solver and ``three_d`` the sparse D3Q6x12 solver.  The time step
runs in ``libcvlbm.so`` (hand-written CUDA for sm_100a) on PyTorch CUDA
buffers.
"""

__version__ = "1.0.0"
