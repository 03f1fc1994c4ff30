"""B200-native SVPF step engine (host side).

The directory name is not a Python identifier; load it with
``__graft_entry__.load_package()`` (registers it as ``svpf_b200``).
"""
from .svpf import (SVPF, Batch, Config, Ctl, Out, Params, SVPFResult, autotune, build_info,  # noqa: F401
                   default_config, lib, philox, pipe_rates, LIB_PATH, CONFIG_FIELDS, production_config, Grad,
                   grad_config, Stream, FusedV2, MultiScale, Estimator)
