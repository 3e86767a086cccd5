"""B200-native engine for zxtalori's QVM repulsion path: orientation samples on SO(3)/K
relaxed by Quey-Villani-Maurice geodesic repulsion with Barzilai-Borwein steps, their pair
measures and the nearest-neighbour spacing pass, on hand-written sm_100a CUDA kernels."""
__version__ = "0.3.0"
from .api import GROUPS, PRECISIONS, Grid, from_quaternions, generate, haar, load, library_path

__all__ = ["GROUPS", "PRECISIONS", "Grid", "generate", "from_quaternions", "load", "haar", "library_path"]
