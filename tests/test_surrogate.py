"""The FDTD-trained surrogate: labels from the batched FDTD agree with the
single-grid solver, training on FDTD data gains over the no-network answer
on held-out designs, and ``forward`` keeps the reference's periodic
full-solver correction."""

from __future__ import annotations

import pytest
import torch

from conftest import rel_l2


@pytest.mark.gpu
def test_labels_match_single_grid_solver(cuda):
    from diffnano_b200.solvers import FDTDSolver2D
    from diffnano_b200.surrogate.data import FDTDLabeler, TMzSetup, blob_designs, design_eps
    setup = TMzSetup()
    lab = FDTDLabeler(setup, chunk=4, device=cuda)
    masks, _ = blob_designs(3, seed=5, device=cuda)
    eps_d = design_eps(masks)
    labels = lab.label(eps_d)
    solver = FDTDSolver2D(grid_shape=(setup.side, setup.side), dl=setup.dl,
                          wavelength_nm=setup.center_nm, pml_layers=setup.pml,
                          n_steps=setup.n_steps, courant=setup.courant, device=cuda,
                          dtype=torch.float32,
                          monitors=[{"component": "Ez", "row": setup.mon_row,
                                     "wavelengths_nm": list(setup.wavelengths_nm)}])
    src = setup.instance().source
    eps_full = lab.full_eps(eps_d)
    for i in range(3):
        r = solver.forward(eps_full[i], source=dict(src))
        mon = r.metadata["monitors"][0]["dft"]
        ref = mon[..., setup.offset:setup.offset + setup.design].reshape(labels[i].shape)
        assert rel_l2(labels[i], ref) < 1e-5


@pytest.mark.gpu
def test_trained_surrogate_gains_over_no_network(cuda):
    from diffnano_b200.surrogate.data import FDTDLabeler, TMzSetup, make_dataset
    from diffnano_b200.surrogate.surrogate import FNOSurrogate
    lab = FDTDLabeler(TMzSetup(), chunk=2048, device=cuda)
    designs, labels = make_dataset(4096, seed=3, labeler=lab)
    test_d, test_l = make_dataset(256, seed=4, labeler=lab)
    sur = FNOSurrogate(lab, batch_size=256, lr=1e-3, device=cuda, seed=0)
    hist = sur.train_surrogate(n_epochs=20, designs=designs, labels=labels)
    assert hist[-1] < 0.5 * hist[0], hist
    acc = sur.accuracy(designs=test_d, labels=test_l)
    print(acc)
    # the no-network answer is the mean training field
    assert acc["mean_rel_l2"] < 0.9 * acc["mean_predictor_rel_l2"], acc


@pytest.mark.gpu
def test_forward_periodic_correction(cuda):
    from diffnano_b200.surrogate.data import FDTDLabeler, TMzSetup, make_dataset
    from diffnano_b200.surrogate.surrogate import FNOSurrogate
    lab = FDTDLabeler(TMzSetup(), chunk=64, device=cuda)
    designs, labels = make_dataset(64, seed=8, labeler=lab)
    sur = FNOSurrogate(lab, batch_size=32, correction_interval=3, device=cuda)
    sur.train_surrogate(n_epochs=1, designs=designs, labels=labels)
    flags = [sur.forward(designs[i]).metadata["surrogate"] for i in range(6)]
    assert flags == [True, True, False, True, True, False]
    r = sur.forward(designs[0])
    assert r.field.shape == (1, 3, 128) and r.field.dtype == torch.complex128
    assert sur.stats["total_corrections"] == 2
    with pytest.raises(ValueError):
        sur.forward(designs[0], wavelengths=[1234.0])
