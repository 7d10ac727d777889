"""h2factory_b200: the H2 matrix-vector product of H2Factory.jl on NVIDIA B200.

The package directory is `h2factory.jl_b200/`; it is imported as `h2factory_b200`.

* `trees`    -- 2^D trees and the flattened H2Trees-style plans (host side);
* `methods`  -- interpolation FMM method data (Chebyshev / equispaced-Toeplitz, Laplace /
                Helmholtz): what an H2Factory method supplies;
* `core`     -- H2Core (read-only map data), DeviceCore, H2Workspace, mul_/farmul_/nearmul_,
                transpose/adjoint views: H2Factory's map API over the C ABI;
* `_abi`     -- ctypes mirror of include/h2b200.h and the library loader;
* `autotune` -- per-shape choice of the serving block width and requests in flight, cached;
* `build`    -- compiles csrc/ into libh2b200.so (sm_100a).
"""

from . import trees, _abi  # noqa: F401
from .core import (H2Core, DeviceCore, H2Workspace, OrientedMap, adjoint, farmul_, flatten,  # noqa: F401
                   map_blob, mul_, nearmul_, profilemul, read_blob, save_map, similarworkspace,
                   transpose)
from . import methods  # noqa: F401
from . import batch  # noqa: F401
from . import autotune  # noqa: F401
from ._abi import (H2B_ADJOINT as ADJOINT, H2B_FORWARD as FORWARD,  # noqa: F401
                   H2B_TRANSPOSE as TRANSPOSE, H2BError, WorkspaceBusyError)
