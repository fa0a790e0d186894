"""CPU-side checks of the C-ABI library: it loads without a GPU and exports every symbol
declared in include/*.h (no compute call is made here)."""
import ctypes
import os
import re

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    inc = os.path.join(REPO, "include")
    for f in sorted(os.listdir(inc)):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(inc, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", text, re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof"):
                names.append(name)
    return sorted(set(names))


def test_header_parses():
    names = declared_functions()
    for must in ("write_custom_commit", "commit_witness", "calculate_const_tree", "set_hash_family",
                 "gen_device_buffers", "get_stream_proofs", "b200_commit_device", "b200_lde_device"):
        assert must in names


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_symbol(pkg):
    assert set(declared_functions()) <= set(pkg.exported_symbols())


def test_host_only_calls_without_gpu(pkg):
    # pure host computations, no device work
    assert pkg.tree_num_elements(1 << 17, 4) == 699060
    assert pkg.tree_num_elements(1, 4) == 4
    assert pkg.lde_scratch_words(10, 3) == 3 << 10
    import oracle
    for n in (1, 2, 3, 5, 17, 1000):
        for ar in (2, 3, 4):
            assert pkg.tree_num_elements(n, ar) == oracle.tree_num_elements(n, ar)


def test_synthetic_generator_host(pkg):
    import numpy as np
    a = pkg.fill_random_host(1000, 3)
    b = pkg.fill_random_host(1000, 3)
    c = pkg.fill_random_host(1000, 4)
    assert (a == b).all() and not (a == c).all()
    assert (a < np.uint64(0xFFFFFFFF00000001)).all()


def test_product_does_not_reference_oracle():
    """The shipped library and its Python mirror never load the CPU checkers."""
    pkgdir = os.path.join(REPO, "pil2-proofman_b200")
    for root, _, files in os.walk(pkgdir):
        for f in files:
            # the constant-table generators are build-time scripts that say who includes their output
            if f.endswith((".py", ".cu", ".cuh", ".h")) and not f.startswith("gen_poseidon"):
                text = open(os.path.join(root, f)).read()
                assert "oracle" not in text, f
                assert "libpil2ref" not in text and "gl_oracle" not in text, f


def test_kernel_names_list_every_kernel(pkg):
    """b200_kernel_names() (the launch evidence the library reports) names every __global__ kernel
    defined in its sources, and nothing else."""
    import glob
    import re
    defs = set()
    for f in glob.glob(os.path.join(REPO, "pil2-proofman_b200", "csrc", "*.cu*")):
        text = open(f).read()
        for m in re.finditer(r"__global__\s+void\s+(?:__launch_bounds__\((?:[^()]|\([^()]*\))*\)\s*)?(\w+)\s*\(", text):
            defs.add(m.group(1))
    names = set(pkg.load().b200_kernel_names().decode().split())
    assert defs == names, (sorted(defs - names), sorted(names - defs))
