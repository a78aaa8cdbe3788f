"""mpifield_b200: mpifield's particle-grid hot path on one B200, as a kernel backend.

B-spline gather and scatter of degree 0-3 in 1D-3D (`LINEAR`, `QUADRATIC`, `CUBIC`), the
charge-conserving path deposit (`WHITNEY`, `QUADRATIC_EDGES`, `CUBIC_EDGES`), the halo
fill and fold-back on one GPU and between the ranks of a split field (`HaloExchange`),
behind mpifield's `Weighting` / `EdgeWeighting`
kernel convention and a `Field` with its gather / scatter / deposit_density; device
arrays of any producer (CuPy, torch, ``__cuda_array_interface__``, DLPack) on the
caller's stream, hand-written sm_100a kernels through the C ABI of
``include/mpifield_b200.h`` (``libmpifield_b200.so``). There is no CPU fallback.
"""

from mpifield_b200._arrays import use_stream
from mpifield_b200._types import BlockGrid, Bounds
from mpifield_b200.edges import CUBIC_EDGES, QUADRATIC_EDGES, WHITNEY, EdgeWeighting
from mpifield_b200.exchange import Decomposition, HaloExchange
from mpifield_b200.field import Field
from mpifield_b200.kernels import KERNELS
from mpifield_b200.sorting import TileOrder, permute, resort_by_tile, sort_by_tile, unpermute
from mpifield_b200.splines import CLAMPED_SPLINES, SPLINES, Splines, splines
from mpifield_b200.weighting import CUBIC, LINEAR, QUADRATIC, Weighting, spline_weighting

__all__ = [
    "BlockGrid", "Bounds", "CLAMPED_SPLINES", "CUBIC", "CUBIC_EDGES", "Decomposition", "EdgeWeighting", "Field",
    "HaloExchange", "KERNELS",
    "LINEAR", "QUADRATIC", "QUADRATIC_EDGES", "SPLINES", "Splines", "TileOrder", "WHITNEY", "Weighting",
    "permute", "resort_by_tile", "sort_by_tile", "spline_weighting", "splines", "unpermute", "use_stream",
]
__version__ = "1.0.0"
