"""The bounds-checked build (RESTIR_CHECKS=1, restir_b200/librestir_gpu_checked.so),
the stand-in for a memory checker: every BVH row and light-list row index is
tested before its load, and one out of range raises status bit 4 instead of
reading outside the buffer. Run in a process of its own (the library is
chosen when restir_b200 loads), frames of two configurations must equal the
oracle bit for bit, as with the product build, with no index out of range."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
CHECKED = ROOT / "restir_b200" / "librestir_gpu_checked.so"

SCRIPT = r"""
import json, sys
sys.path.insert(0, {root!r})
import restir_b200 as rb
from oracle.frame import run_checked
from tests.helpers import make_scene
out = {{}}
for name, (scene, size, overrides) in {{
        "courtyard": ((rb.SCENE_COURTYARD, 0, 100000), (192, 108), dict(extra_lights=64)),
        "bvh-rays": ((rb.SCENE_CORNELL, 0, 0), (64, 64), dict(gi_divisor=1, ray_mode=rb.RAY_BVH, initial_candidates=4)),
        }}.items():
    setup = make_scene(*scene, extra_lights=overrides.get("extra_lights", 0))
    settings = setup.settings
    for k, v in overrides.items():
        setattr(settings, k, v)
    settings.grid_mode = rb.GRID_DETERMINISTIC
    if "extra_lights" in overrides:
        setup.lights = rb.Lights(setup.bvh, setup.mesh, settings)
    rb.status_flags()
    report, _, _ = run_checked(setup, size[0], size[1], 3, settings, gi_wavefront=True)
    out[name] = {{"report": report, "status": rb.status_flags()}}
out["library"] = str(rb.LIBRARY_PATH)
print(json.dumps(out))
"""


@pytest.mark.gpu
def test_bounds_checked_build_matches_the_oracle_with_no_index_out_of_range():
    if not CHECKED.exists():
        subprocess.run([sys.executable, "-m", "restir_b200.build", "--checks"], cwd=ROOT, check=True)
    env = dict(os.environ, RESTIR_LIBRARY=str(CHECKED))
    result = subprocess.run([sys.executable, "-c", SCRIPT.format(root=str(ROOT))], cwd=ROOT, env=env,
                            capture_output=True, text=True, timeout=900)
    assert result.returncode == 0, result.stderr[-2000:]
    out = json.loads(result.stdout.strip().splitlines()[-1])
    assert out["library"].endswith("librestir_gpu_checked.so")
    for name in ("courtyard", "bvh-rays"):
        assert out[name]["report"] == {}, (name, out[name])
        assert out[name]["status"] & 16 == 0, (name, out[name])
