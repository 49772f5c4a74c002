"""Restart checkpoints (nova_checkpoint_write / nova_checkpoint_read): a
lossless FP64 copy of a state.  A run restarted from a checkpoint must
continue bit for bit like the run that wrote it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nova():
    from novaclone_b200 import nova
    return nova


def ns_state(nova, M, prec, seed=0):
    U0 = 0.3 * np.random.default_rng(seed).standard_normal((3,) + M.shape)
    return nova.Field(M, 3, prec).upload_soa(U0), nova.Field(M, 1)


def test_round_trip_and_bitwise_restart(nova, tmp_path):
    M = nova.Mesh((16, 12, 8), L=(2 * np.pi, 2.0, 3.0))
    rd = nova.run_desc(model="ns", dt=2e-3, nu=0.01)
    U, p = ns_state(nova, M, nova.F64)
    nova.advance(M, rd, U, p, nsteps=3)
    path = str(tmp_path / "s3.nova")
    nova.checkpoint_write(M, path, U, p, t=0.006, step=3)
    U2, p2 = nova.Field(M, 3), nova.Field(M, 1)
    t, step = nova.checkpoint_read(M, path, U2, p2)
    assert (t, step) == (0.006, 3)
    assert np.array_equal(U2.download_soa(), U.download_soa())
    assert np.array_equal(p2.download_soa(), p.download_soa())
    nova.advance(M, rd, U, p, nsteps=2)
    nova.advance(M, rd, U2, p2, nsteps=2)
    assert np.array_equal(U2.download_soa(), U.download_soa())


def test_split_fields_keep_their_48_bits(nova, tmp_path):
    M = nova.Mesh((16, 16, 32))
    U, p = ns_state(nova, M, nova.F32SPLIT, seed=1)
    nova.advance(M, nova.run_desc(model="ns", precision=nova.F32SPLIT, dt=2e-3, nu=0.01), U, p, nsteps=2)
    path = str(tmp_path / "split.nova")
    nova.checkpoint_write(M, path, U, p)
    U2 = nova.Field(M, 3, nova.F32SPLIT)
    U64 = nova.Field(M, 3)
    nova.checkpoint_read(M, path, U=U2)
    nova.checkpoint_read(M, path, U=U64)
    ref = U.download_soa()
    assert np.array_equal(U64.download_soa(), ref)
    assert np.abs(U2.download_soa() - ref).max() <= 1e-15 * np.abs(ref).max()


def test_wall_bcs_and_mhd_state_travel_with_the_fields(nova, tmp_path):
    M = nova.Mesh((16, 12, 8), L=(2 * np.pi, 2 * np.pi, np.pi), walls=(0, 1, 0))
    U = nova.Field(M, 3).upload_soa(np.random.default_rng(2).standard_normal((3,) + M.shape))
    types, vals = [0] * 18, [0.0] * 18
    for face, (ty, v) in ((0, (2, 0.5)), (1, (1, -0.25))):  # north Dirichlet 0.5, south Neumann -0.25 on u
        types[face], vals[face] = ty, v
    for c in (1, 2):
        for face in (0, 1):
            types[face + 6 * c], vals[face + 6 * c] = 1, 0.0
    U.set_bc(types, vals)
    path = str(tmp_path / "walls.nova")
    nova.checkpoint_write(M, path, U)
    V = nova.Field(M, 3)
    nova.checkpoint_read(M, path, U=V)
    assert np.array_equal(V.download(), U.download())  # ghosts from the restored BCs

    Mm = nova.Mesh((16, 16, 16))
    rng = np.random.default_rng(3)
    fs = [nova.Field(Mm, nc).upload_soa(rng.standard_normal((nc,) + Mm.shape)) for nc in (3, 1, 3, 1)]
    path = str(tmp_path / "mhd.nova")
    nova.checkpoint_write(Mm, path, *fs, t=1.5, step=7)
    gs = [nova.Field(Mm, nc) for nc in (3, 1, 3, 1)]
    assert nova.checkpoint_read(Mm, path, *gs) == (1.5, 7)
    for f, g in zip(fs, gs):
        assert np.array_equal(f.download_soa(), g.download_soa())


def test_a_checkpoint_of_another_mesh_is_refused(nova, tmp_path):
    M = nova.Mesh((16, 12, 8))
    U, p = ns_state(nova, M, nova.F64)
    path = str(tmp_path / "a.nova")
    nova.checkpoint_write(M, path, U, p)
    other = nova.Mesh((16, 12, 10))
    with pytest.raises(nova.NovaError) as e:
        nova.checkpoint_read(other, path, nova.Field(other, 3))
    assert e.value.status == nova.E_INVALID
    with pytest.raises(nova.NovaError) as e:
        nova.checkpoint_read(M, str(tmp_path / "missing.nova"), U)
    assert e.value.status == nova.E_INVALID


def test_ensight_field_round_trip(nova, tmp_path):
    """nova_ensight_write_field / read_field: the reference's float32 restart path."""
    M = nova.Mesh((16, 12, 8), walls=(0, 1, 0))
    x = np.random.default_rng(4).standard_normal((3,) + M.shape)
    U = nova.Field(M, 3).upload_soa(x)
    nova.ensight.write_field(U, str(tmp_path), "U", 3)
    V = nova.ensight.read_field(nova.Field(M, 3), str(tmp_path), "U", 3)
    assert np.array_equal(V.download_soa(), x.astype(np.float32).astype(np.float64))
