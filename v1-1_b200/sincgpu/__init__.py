"""sincgpu: B200 (sm_100a) sinc-DVR orbital right-hand side behind a C ABI.

Host-side mirror of the reference's SINCDVR project interface
(SINCDVR/coreproject.f90, MCTDH.SRC/mean.f90, MCTDH.SRC/derivs.f90): the
methods of :class:`SincProject` keep the reference routine names, argument
meaning and Fortran array layouts, and call the CUDA library through its
``extern "C"`` entry points (include/sincgpu.h).  There is no CPU fallback:
if libsincgpu.so is missing or no CUDA device is present, calls fail.
"""
from .capi import (  # noqa: F401
    Batch,
    SincGpuError,
    SincProject,
    load_library,
    library_path,
    exported_symbols,
)
from .walks import WalkTables  # noqa: F401,E402
