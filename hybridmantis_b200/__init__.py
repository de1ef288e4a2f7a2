"""fd2-b200: B200-native fastDETECT2 (optical-photon transport in columnar CsI).

The product is the C ABI in ``lib/libfd2.so`` (header ``include/fd2.h``);
this package is its Python host layer.  Build with ``make -C hybridmantis_b200``.
"""
from ._lib import Fd2Error, load  # noqa: F401
from .fastdetect2 import (COUNT_GAUSSIAN, COUNT_GIVEN, COUNT_POISSON, REPLAY_FP64, REPLAY_REF,  # noqa: F401
                          UNITS_CM, UNITS_UM, EventSet, Ingest, OpticalTransport, default_params, params_to_geometry, prf_dims,
                          read_events_binary, read_events_text, read_input_file, synth_events,
                          write_events_binary, write_events_text, write_output_files)
from .surrogate import Surrogate  # noqa: F401,E402
from .xray import Material as XrayMaterial, XrayFrontEnd  # noqa: F401,E402
