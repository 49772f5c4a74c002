"""nova_field_maxabs_noalloc, the allocation-free max|s| (static device scratch),
against nova_field_maxabs on the same fields.  The maximum of absolute values
is exact in any reduction order, so the tolerance is a relative 1e-15.  This
file is collected last so that it also runs after every other GPU test in one
process."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-15
MAX_NODES = 1 << 27  # NOVA_MAXABS_NOALLOC_MAX_NODES


@pytest.fixture(scope="module")
def nova():
    from novaclone_b200 import nova
    return nova


def scalar(nova, mesh, values):
    return nova.Field(mesh, 1).upload_soa(values[None])


def test_two_calls_in_a_row_match_the_allocating_entry_point(nova):
    N = (24, 20, 28)
    M = nova.Mesh(N)
    rng = np.random.default_rng(21)
    a = rng.standard_normal(N)
    b = 0.25 * rng.standard_normal(N)   # smaller maximum: a stale result would show
    fa, fb = scalar(nova, M, a), scalar(nova, M, b)
    got = [nova.tools.maximum_noalloc(fa), nova.tools.maximum_noalloc(fb)]
    want = [nova.tools.maximum(fa), nova.tools.maximum(fb)]
    for g, w, x in zip(got, want, (a, b)):
        assert g == pytest.approx(w, rel=TOL, abs=0.0)
        assert g == pytest.approx(np.abs(x).max(), rel=TOL, abs=0.0)
    assert got[1] < got[0]


@pytest.mark.parametrize("N,walls", [((33, 17, 40), (0, 0, 0)), ((64, 64, 64), (0, 0, 0)),
                                     ((16, 12, 8), (0, 1, 0))])
def test_ragged_chunks_and_wall_rows(nova, N, walls):
    """The last chunk of 16384 nodes is partial; the maximum sits in its final
    node (and, with y walls, in the north wall row)."""
    M = nova.Mesh(N, L=(2 * np.pi, 2 * np.pi, np.pi), walls=walls)
    x = np.random.default_rng(3).uniform(-1.0, 1.0, M.shape)  # stored nodes (N1+1 rows with walls)
    x[-1, -1, -1] = -7.5
    f = scalar(nova, M, x)
    for _ in range(2):
        assert nova.tools.maximum_noalloc(f) == 7.5
        assert nova.tools.maximum(f) == 7.5


def test_repeated_calls_leave_device_memory_unchanged(nova):
    import torch
    N = (32, 32, 32)
    warm = nova.Mesh(N)
    nova.tools.maximum_noalloc(scalar(nova, warm, np.ones(N)))  # the device code is loaded
    M = nova.Mesh(N)
    f = scalar(nova, M, np.linspace(-3.0, 2.0, np.prod(N)).reshape(N))
    free0 = torch.cuda.mem_get_info(0)[0]
    vals = [nova.tools.maximum_noalloc(f) for _ in range(3)]
    assert torch.cuda.mem_get_info(0)[0] == free0
    assert vals == [3.0, 3.0, 3.0]


def test_fields_beyond_the_static_scratch_are_refused(nova):
    N = (513, 512, 512)
    assert N[0] * N[1] * N[2] > MAX_NODES
    M = nova.Mesh(N)
    f = nova.Field(M, 1)
    with pytest.raises(nova.NovaError) as e:
        nova.tools.maximum_noalloc(f)
    assert e.value.status == nova.E_INVALID
    assert "NOVA_MAXABS_NOALLOC_MAX_NODES" in str(e.value)
    del f
