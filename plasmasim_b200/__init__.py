"""B200-native (sm_100a) 3D particle-in-cell step of PLASMAsim's PIC/3d_pic458_domain.c."""
from .pic3d import (BOTH, ELECTRON, ION, GRID_FIELDS, Pic3D, PicConfig, PicError,  # noqa: F401
                    load_library)
