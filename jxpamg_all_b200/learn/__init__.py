"""Learned AMG settings for the mixed-precision CPR path.

A 16 -> 64 (tanh) -> 3 MLP maps cheap statistics of each AMG level operator
(jxcpr_solver_level_features) to that level's strength threshold and the
interval of its degree-3 Chebyshev smoother.  ``datagen`` produces training
data by solving seeded reservoir systems with a grid of candidate settings,
``train`` fits the network with the library's own CUDA forward / backward /
Adam kernels (jxcpr_mlp_*) and writes the weights compiled into the library.
"""
from .model import (  # noqa: F401
    N_IN, N_HIDDEN, N_OUT, N_WEIGHTS, lower_of, theta_of, upper_of, to_logits, pack, unpack, write_weights_inc,
)
