"""The C ABI surface: the library loads without a GPU and exports every symbol include/ks_cuda.h
declares; the Python binding names the same set. No compute call here (CPU-only)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ks_cuda.h")
LIB = os.path.join(ROOT, "atomic-sandbox_b200", "libks_b200.so")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ks_[a-z0-9_]+)\s*\(", text)) - {"ks_abort_fn"})


def test_header_declares_the_solver_entry_points():
    names = declared()
    for must in ("ks_solver_create", "ks_solver_destroy", "ks_solve", "ks_forces", "ks_last_error", "ks_state_evals",
                 "ks_hpsi_device"):
        assert must in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        import ks_b200
        ks_b200.build()
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_binding_lists_the_same_symbols(ks):
    assert sorted(ks.EXPORTED) == declared()


def test_pitch_is_host_only(ks):
    # ks_field_pitch needs no device: multiples of 4 floats (16-byte TMA strides)
    for n in (5, 33, 48, 95, 96, 128):
        p = ks.field_pitch(n)
        assert p >= n and p % 4 == 0 and p - n < 4


def test_spin_split_matches_reference_rules(ks):
    # crates/qm/src/scf.rs:1151-1160 (spin_counts)
    assert ks.spin_split(1) == (1, 0)
    assert ks.spin_split(3) == (2, 1)
    assert ks.spin_split(2, 3) == (2, 0)
    assert ks.spin_split(0) == (0, 0)


def _count_params(sig):
    sig = sig.strip()
    if sig in ("", "void"):
        return 0
    depth, n = 0, 1
    for ch in sig:
        if ch in "(<[":
            depth += 1
        elif ch in ")>]":
            depth -= 1
        elif ch == "," and depth == 0:
            n += 1
    return n


def test_rust_binding_declares_every_symbol():
    """The Rust sys crate (rust/qm-b200-sys/src/lib.rs) declares every entry point of the header in its extern block,
    each with the header's parameter count."""
    header = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    doc = open(os.path.join(ROOT, "rust", "qm-b200-sys", "src", "lib.rs")).read()
    block = doc[doc.index('extern "C" {'):]
    block = block[:block.index("\n}\n")]
    seen, wrong = 0, []
    for m in re.finditer(r"\b(ks_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", header):
        name, args = m.group(1), m.group(2)
        r = re.search(r"pub fn " + name + r"\((.*?)\)\s*(->|;)", block, flags=re.S)
        if not r:
            wrong.append((name, "not declared"))
        elif _count_params(args) != _count_params(r.group(1)):
            wrong.append((name, _count_params(args), _count_params(r.group(1))))
        seen += 1
    assert seen == len(declared()), (seen, len(declared()))
    assert not wrong, wrong
