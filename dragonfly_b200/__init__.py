"""dragonfly_b200: duaneloh/Dragonfly's EMC iteration on an NVIDIA B200.

The same public names as the reference package (dragonfly/__init__.py:1-7);
EMCRecon lives in dragonfly_b200.recon as in the reference. The iteration runs
in libdfgpu.so (sm_100a CUDA behind the C ABI in include/dragonfly_b200.h);
importing the package does not need a GPU, running an iteration does.
"""
from .detector import Detector, CDetector
from .emcfile import EMCReader, EMCWriter, CDataset
from .quaternion import Quaternion
from .model import Model
from .params import EMCParams
from .iterate import Iterate

__all__ = ["Detector", "CDetector", "EMCReader", "EMCWriter", "CDataset", "Quaternion", "Model", "EMCParams",
           "Iterate"]
