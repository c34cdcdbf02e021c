"""What the trained radiance cache gains over the method without it.

The cache-only GI form (restir_gi_from_cache: the network's radiance at each
GI pixel's surface, no GI rays) is run three ways on the same seeded
courtyard view, each against the FP64 progressive reference of that view
(the reference renderer: the plain estimator with every shortcut off):

  * trained: the network trained online on the path suffixes the renderer
    traces (the default learning rate);
  * untrained: the same network and the same frames, with a learning rate of
    1e-30, so its weights and hash table stay at their seeded start;
  * no GI: the plain method with its GI turned off (no candidates, no
    reuse, no specular GI), the cost class of the cache-only form.

The trained network must lower the relative MSE against the reference well
below both: the indirect light it supplies is learned, not an artefact of
its start or of leaving GI out.
"""
import numpy as np
import pytest

import restir_b200 as rb

WIDTH, HEIGHT = 320, 180
REFERENCE_FRAMES = 256
TRAIN_FRAMES = 150
ERROR_FRAMES = 60


def run_form(mesh, changes: dict) -> float:
    settings = rb.default_settings(mesh)
    for name, value in changes.items():
        setattr(settings, name, value)
    renderer = rb.Renderer(settings)
    renderer.set_scene(mesh, use_scene_defaults=True)
    frame = rb.frame_input(mesh, WIDTH, HEIGHT)
    renderer.set_reference_accumulation(True)
    for _ in range(REFERENCE_FRAMES):
        renderer.render(frame)
    renderer.set_reference_accumulation(False)
    for _ in range(TRAIN_FRAMES):
        renderer.render(frame)
    errors = []
    for _ in range(ERROR_FRAMES):
        renderer.render(frame)
        metrics = renderer.frame_submitted()
        assert metrics.valid and metrics.reference_frames == REFERENCE_FRAMES
        errors.append(metrics.relative_mse)
    renderer.close()
    return float(np.mean(errors))


@pytest.mark.gpu
def test_trained_cache_lowers_the_error_of_the_cache_only_gi():
    mesh = rb.Mesh.procedural(rb.SCENE_COURTYARD, 0, 20000)
    cache_only = {"radiance_cache": 1, "cache_only_gi": 1, "specular_gi": 0, "cache_training_samples": 16384}
    rb.status_flags()
    trained = run_form(mesh, cache_only)
    untrained = run_form(mesh, dict(cache_only, cache_learning_rate=1e-30))
    no_gi = run_form(mesh, {"initial_candidates": 0, "temporal_taps": 0, "spatial_taps": 0, "specular_gi": 0})
    plain = run_form(mesh, {"specular_gi": 0})
    print(f"relMSE vs FP64 reference: trained cache {trained:.4f}, untrained cache {untrained:.4f}, "
          f"no GI {no_gi:.4f}, plain method {plain:.4f}")
    assert rb.status_flags() & 8 == 0
    assert np.isfinite([trained, untrained, no_gi, plain]).all()
    assert trained < 0.8 * untrained
    assert trained < 0.8 * no_gi
