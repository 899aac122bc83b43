"""Test infrastructure: the CPU restatement of the reference's path-tracing
routines (ffo), the reference's own routines compiled for the host (ffref,
ffrefcuda) and the recipes that build them.  Only the tests, the smoke check
and the benchmark's CPU-baseline legs use it, as the checker."""
import os
from pathlib import Path

# The reference checkout the recipes under oracle/ build from; machines that
# only run the prebuilt libraries do not have it.
REF_DIR = Path(os.environ.get("FF_REF_DIR", "/root/reference/CUDA-RayTracer"))
