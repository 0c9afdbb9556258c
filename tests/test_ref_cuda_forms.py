"""Which float form of `ex*ex + ey*ey` does the reference CUDA build use?

Settled by black-box label tests only (no reading of compiled code): the
probe families of probes.py are clustered by the reference's own CUDA path
(oracle/_ref/cuda, built from its sources with its own flags), and every
assignment of forms to the family's call sites is replayed in the oracle.
The oracle's REFERENCE_FORMS must reproduce the reference's labels slot for
slot, and the product must produce the same labels.
"""

import itertools

import numpy as np
import pytest
import torch

import oracle
import probes
import refmod
from dbscan_torch import dbscan2d

pytestmark = pytest.mark.gpu

FORM_NAMES = {0: "unfused", 1: "fma(ex,ex,ey*ey)", 2: "fma(ey,ey,ex*ex)"}


def _consistent(fam, X, eps, ms, slot, want_sig):
    sites = probes.SITES_OF[fam]
    ok = []
    for combo in itertools.product((0, 1, 2), repeat=len(sites)):
        forms = list(oracle.REFERENCE_FORMS)
        for s, f in zip(sites, combo):
            forms[s] = f
        sig = probes.slot_signature(oracle.dbscan2d(X, eps, ms, forms=forms), slot)
        if np.array_equal(sig, want_sig):
            ok.append(tuple(FORM_NAMES[f] for f in combo))
    return ok


@pytest.mark.parametrize("fam", list(probes.FAMILIES))
def test_reference_forms(fam):
    ref = refmod.load("cuda")
    if ref is None:
        pytest.skip("reference CUDA build not present in oracle/_ref/cuda")
    X, eps, ms, slot, _ = probes.FAMILIES[fam]()
    want = ref.dbscan2d(torch.from_numpy(X).cuda(), eps, ms).cpu().numpy()
    want_sig = probes.slot_signature(want, slot)
    got = oracle.dbscan2d(X, eps, ms)
    got_sig = probes.slot_signature(got, slot)
    bad = np.flatnonzero((got_sig != want_sig).any(1))
    if bad.size:
        ok = _consistent(fam, X, eps, ms, slot, want_sig)
        pytest.fail(f"{fam}: REFERENCE_FORMS disagrees with the reference on {bad.size} slots; "
                    f"site forms consistent with the reference: {ok}")


@pytest.mark.parametrize("fam", list(probes.FAMILIES))
def test_product_matches_reference_on_probes(fam):
    X, eps, ms, slot, _ = probes.FAMILIES[fam]()
    ours = dbscan2d(torch.from_numpy(X).cuda(), eps, ms).cpu().numpy()
    assert np.array_equal(ours, oracle.dbscan2d(X, eps, ms))
    ref = refmod.load("cuda")
    if ref is not None:
        want = ref.dbscan2d(torch.from_numpy(X).cuda(), eps, ms).cpu().numpy()
        assert np.array_equal(ours, want)
