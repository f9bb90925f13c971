"""B200-native LiteRT ray query (BVHRT::RayQuery_NearestHit) behind the CrossRT
ISceneObject API.  The compute path is liblrt_b200.so (sm_100a CUDA); this
package only binds it (lrt.py), mirrors its C structs (_abi.py), builds it
(build.py) and generates benchmark workloads (workloads.py)."""
from ._abi import (BUILD_HIGH, BUILD_LOW, BUILD_MEDIUM, BUILD_REFIT, HIT_DTYPE, LIGHT_AMBIENT,  # noqa: F401
                   LIGHT_DIRECT, LIGHT_DTYPE, LIGHT_POINT, MATERIAL_COLORED, MATERIAL_DTYPE, MATERIAL_TEXTURED,
                   Camera, Preset, default_preset, parity_preset)
from .lrt import LrtError, SceneRT, lib  # noqa: F401
