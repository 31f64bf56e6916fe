"""What the trained leverage model gains over the method without it: on held-out mixture instances (seeds
outside the training range), the Nystrom factor on r landmarks drawn by the committed model has a lower sampled
residual ||Q - Z Z^T||_F / ||Q||_F than on r landmarks drawn uniformly (the same Gumbel top-k with all scores
equal), averaged over three instances."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_learned_landmarks_beat_uniform(gpu_ctx):
    from darray_optimizer_b200 import landmarks
    net = landmarks.load_model(gpu_ctx)
    res = landmarks.evaluate(gpu_ctx, net, seeds=(90_011, 90_012, 90_013), r=512)
    learned = np.array([r["learned"] for r in res])
    uniform = np.array([r["uniform"] for r in res])
    print("learned", learned, "uniform", uniform)
    assert np.all(learned < 1.0) and np.all(uniform < 1.0)
    assert learned.mean() < 0.98 * uniform.mean()
