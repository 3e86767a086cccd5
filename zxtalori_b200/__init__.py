"""B200-native engine for zxtalori's QVM repulsion path: orientation samples on SO(3)/K
relaxed by Quey-Villani-Maurice geodesic repulsion with Barzilai-Borwein steps, their pair
measures and the nearest-neighbour spacing pass, on hand-written sm_100a CUDA kernels."""
__version__ = "0.3.0"
import os as _os

# Samples relax side by side on their own CUDA streams; more hardware queues than the
# default 8 keep streams that share one from waiting on each other. Read by the driver
# when CUDA initialises, so it must be set before the first CUDA call of the process.
_os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from .api import GROUPS, PRECISIONS, Grid, from_quaternions, generate, haar, hopf_points, load, library_path  # noqa: E402

__all__ = ["GROUPS", "PRECISIONS", "Grid", "generate", "from_quaternions", "load", "haar", "hopf_points", "library_path"]
