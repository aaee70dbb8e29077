"""The Fluent mesh reader (``gputest_b200.mesh.fluent``), the input step of the path, against the
reference's reader (``flowtrace/mesh/fluent_msh.py``) through the digests of
``tests/golden/fluent_digests.json`` (made by ``tests/golden/make_fluent_golden.py``): every array
and the zone table of what it builds, on the reference's own mesh files and on ASCII and binary
files written here; the writer's round trip; gzip; and the errors of unreadable files. The GPU
test solves a mesh read from a file and the same mesh built in memory."""

import gzip
import json
import os

import numpy as np
import pytest

from gputest_b200.mesh.fluent import FluentMeshError, read_fluent_mesh, write_fluent_mesh
from gputest_b200.mesh.unstructured import cartesian_mesh_2d
from tests.golden.fluent_cases import ARRAYS, digest, generated_cases, generated_meshes

HERE = os.path.dirname(os.path.abspath(__file__))
DIGESTS = json.load(open(os.path.join(HERE, "golden", "fluent_digests.json")))
REFERENCE = os.environ.get("B2S_REFERENCE", "/root/reference")


@pytest.mark.parametrize("key", sorted(DIGESTS["generated"]))
def test_generated_files_read_like_the_reference_reader(tmp_path, key):
    path = generated_cases(str(tmp_path))[key]
    assert digest(read_fluent_mesh(path)) == DIGESTS["generated"][key]


@pytest.mark.parametrize("rel", sorted(DIGESTS["shipped"]))
def test_the_references_mesh_files_read_like_the_reference_reader(rel):
    path = os.path.join(REFERENCE, rel)
    if not os.path.exists(path):
        pytest.skip("the reference's mesh files are not present")
    assert digest(read_fluent_mesh(path)) == DIGESTS["shipped"][rel]


@pytest.mark.parametrize("binary", [False, True])
def test_writer_round_trip_and_gzip(tmp_path, binary):
    for name, m in generated_meshes().items():
        p = tmp_path / f"{name}.msh"
        write_fluent_mesh(m, str(p), binary=binary)
        back = read_fluent_mesh(str(p))
        for k in ARRAYS:
            assert np.array_equal(getattr(back, k), getattr(m, k)), (name, k)
        assert digest(back)["zones"] == digest(m)["zones"]
        gz = read_fluent_mesh(gzip.compress(p.read_bytes()))
        assert digest(gz) == digest(back)


def test_unreadable_files_raise(tmp_path):
    m = generated_meshes()["tri2d"]
    p = tmp_path / "m.msh"
    write_fluent_mesh(m, str(p))
    data = p.read_bytes()
    with pytest.raises(FluentMeshError):
        read_fluent_mesh(data[: len(data) // 2])  # truncated inside a face section
    with pytest.raises(FluentMeshError):
        read_fluent_mesh(b"(0 \"no mesh here\")\n(2 2)\n")
    with pytest.raises(FluentMeshError):
        read_fluent_mesh(data.replace(b"(13 (3 ", b"(13 (3 zz"))  # bad hexadecimal header
    with pytest.raises(FileNotFoundError):
        read_fluent_mesh(str(tmp_path / "missing.msh"))


@pytest.mark.gpu
def test_a_mesh_read_from_a_file_solves_like_the_mesh_it_was_written_from(tmp_path):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gputest_b200.mesh.unstructured import cartesian_mesh_2d
    from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
    from gputest_b200.unstructured.simple import SimpleSolver

    m = cartesian_mesh_2d(24, 24, triangulate="alternating", jitter=0.15, seed=2)
    p = tmp_path / "cavity.msh"
    write_fluent_mesh(m, str(p), binary=True)
    case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, viscosity=0.01,
                            max_iter=30, tol=0.0)
    a, b = SimpleSolver(read_fluent_mesh(str(p)), case), SimpleSolver(m, case)
    a.run()
    b.run()
    for k, v in b.fields().items():
        assert np.array_equal(a.fields()[k], v), k


def test_set_cell_zone_equals_the_reference_and_round_trips_through_a_file(tmp_path):
    """``set_cell_zone`` against digests of the reference's (``tests/golden/cellzone_digests.json``,
    made by ``tests/golden/make_cellzone_golden.py``); its meshes (contiguous cell zones) write and
    read back unchanged, while a mesh whose cell zone is not contiguous is refused by the writer."""
    from gputest_b200.mesh.unstructured import extrude_to_3d, set_cell_zone
    from tests.golden.mesh_cases import cell_zone_cases, with_solid_zone

    ref = json.load(open(os.path.join(HERE, "golden", "cellzone_digests.json")))
    cases = cell_zone_cases(cartesian_mesh_2d, extrude_to_3d, set_cell_zone)
    assert set(cases) == set(ref)
    for key, m in cases.items():
        assert digest(m) == ref[key], key
        p = tmp_path / f"{key}.msh"
        write_fluent_mesh(m, str(p))
        assert digest(read_fluent_mesh(str(p))) == ref[key], key
    scattered, _ = with_solid_zone(cartesian_mesh_2d(8, 6), lambda x: x[:, 1] < 0.5)
    with pytest.raises(ValueError, match="contiguous"):
        write_fluent_mesh(scattered, str(tmp_path / "bad.msh"))
