"""The drop-in adapters through the reference's own interfaces (GPU).

oracle/_ref/adapter_check is built from the reference's unmodified sources
plus encore_b200/adapters/GpuAccel.h and GpuPhotonMap.h (C++98, as the
reference compiles), linked against the engine library.  It calls
AccelerationStructure::build / intersect / update and PhotonMap's
GetNearestNPhotons / GetRadianceEstimate on the reference's Kdtree and
PhotonMap and on the adapters with the same models, rays and photons:

* kd mode: every HitInfo field identical (object, t, point, normal,
  isEntering) on every ray, before and after the scene moves;
* wide-BVH mode: the same primitive, or a tie at the same FP32 t;
* both modes: the batched 8-float call names the per-ray call's primitive,
  and the batched call on the Ray payload (origin, direction) returns the
  8-float batch's hits, field for field;
* photon maps: the same k-nearest photon sets, a valid max-heap as the
  reference returns, radiance within 1e-4 relative.
"""
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
PROG = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "adapter_check"


@pytest.mark.skipif(not PROG.exists(), reason="adapter_check not built (needs the reference sources)")
def test_adapters_match_reference_through_its_interfaces(gpu):
    r = subprocess.run([str(PROG)], capture_output=True, text=True, timeout=600)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out
    assert "result pass" in out, out
