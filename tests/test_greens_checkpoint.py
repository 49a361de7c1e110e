"""Green's function checkpoints (CPU): round trip, loading into another fault-facet order (the
rows and columns follow their facet labels, as tandem's repartitioned restart), partial column
sets, backup of the previous file, and rejection of a different facet set or basis size."""
import os

import numpy as np
import pytest

from tandem_b200.greens import load_checkpoint, save_checkpoint


def _case(nf=5, nbf=3, seed=0):
    rng = np.random.default_rng(seed)
    labels = rng.choice(1000, size=nf, replace=False)
    n = nf * nbf
    G = rng.standard_normal((n, n))
    done = rng.random(n) < 0.6
    G[:, ~done] = 0.0
    return labels, nbf, G, done


def test_round_trip(tmp_path):
    labels, nbf, G, done = _case()
    p = str(tmp_path / "gf.npz")
    save_checkpoint(p, G, done, labels, nbf)
    G2, d2 = load_checkpoint(p, labels, nbf)
    np.testing.assert_array_equal(G2, G)
    np.testing.assert_array_equal(d2, done)


def test_other_facet_order_permutes_blocks(tmp_path):
    labels, nbf, G, done = _case(seed=1)
    p = str(tmp_path / "gf.npz")
    save_checkpoint(p, G, done, labels, nbf)
    perm = np.random.default_rng(2).permutation(len(labels))
    new = labels[perm]
    G2, d2 = load_checkpoint(p, new, nbf)
    # block (i, j) of the new order is block (perm[i], perm[j]) of the old one
    for i in range(len(new)):
        for j in range(len(new)):
            np.testing.assert_array_equal(G2[i * nbf:(i + 1) * nbf, j * nbf:(j + 1) * nbf],
                                          G[perm[i] * nbf:(perm[i] + 1) * nbf, perm[j] * nbf:(perm[j] + 1) * nbf])
        np.testing.assert_array_equal(d2[i * nbf:(i + 1) * nbf], done[perm[i] * nbf:(perm[i] + 1) * nbf])


def test_previous_checkpoint_is_kept_as_backup(tmp_path):
    labels, nbf, G, done = _case(seed=3)
    p = str(tmp_path / "gf.npz")
    save_checkpoint(p, G, done, labels, nbf)
    save_checkpoint(p, 2 * G, done, labels, nbf)
    assert os.path.exists(p + ".bu") and not os.path.exists(p + ".tmp")
    np.testing.assert_array_equal(load_checkpoint(p + ".bu", labels, nbf)[0], G)
    np.testing.assert_array_equal(load_checkpoint(p, labels, nbf)[0], 2 * G)


def test_mismatches_are_rejected(tmp_path):
    labels, nbf, G, done = _case(seed=4)
    p = str(tmp_path / "gf.npz")
    save_checkpoint(p, G, done, labels, nbf)
    with pytest.raises(ValueError, match="different set"):
        load_checkpoint(p, labels + 1, nbf)
    with pytest.raises(ValueError, match="basis functions"):
        load_checkpoint(p, labels, nbf + 1)
