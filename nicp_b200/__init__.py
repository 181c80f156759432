"""nicp_b200 -- B200-native NICP registration (depth -> cloud -> projective ICP).

The compute path is libnicp_b200.so (hand-written sm_100a CUDA behind the C
ABI of include/nicp_gpu.h); this package holds its Python binding, the
reference-named classes (api.py) and the synthetic input generator.
"""
from .api import (AlignerNN, AlignerProjective, Cloud, Context, CorrespondenceFinderNN,  # noqa: F401
                  CorrespondenceFinderProjective,
                  DepthImageConverterIntegralImage, Linearizer, Merger, NormalInformationMatrixCalculator,
                  PinholePointProjector, PointInformationMatrixCalculator, Server, StatsCalculatorIntegralImage,
                  align_batch, build_batch)
