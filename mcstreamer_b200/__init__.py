"""mcstreamer_b200 -- B200-native (sm_100a) implementation of JuMC's electron step.

The compute path is libmcs_b200.so (CUDA kernels behind the C ABI of include/mcs.h);
these Python modules mirror the reference's JuMC / Swarm / MCStreamer call sites on top
of that ABI.  There is no CPU fallback: a missing library raises ImportError on first use.
"""
from . import constants, lxcat  # noqa: F401

__all__ = ["constants", "lxcat", "jumc", "swarm"]
