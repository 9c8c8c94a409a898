"""B200-native (sm_100a) particle-in-cell step of PLASMAsim: the 3D step of
PIC/3d_pic458_domain.c and batched runs of the 2D PIC2D/2d_pic278_mpi.c."""
from .pic3d import (BOTH, ELECTRON, ION, GRID_FIELDS, Pic3D, PicConfig, PicError,  # noqa: F401
                    load_library)
from .pic2d import GRID2D_FIELDS, Pic2DBatch, Pic2DConfig  # noqa: F401,E402
from .decomp import DecomposedPic3D, LocalGroup, NcclTransport, rank_config  # noqa: F401,E402
