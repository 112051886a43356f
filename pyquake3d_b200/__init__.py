"""pyquake3d_b200: PyQuake3D's quasi-dynamic SEAS hot path on NVIDIA B200 (sm_100a).

Host code (this package) mirrors the reference's QDsim / BlockTree call surface and
input formats; all compute runs in libpq3d.so (csrc/, C ABI in include/pq3d.h).
"""
from .mesh import read_mshV2, get_eleVec, write_msh
from .qdsim import QDsim, readPara0

__all__ = ["QDsim", "readPara0", "read_mshV2", "get_eleVec", "write_msh"]
