"""Makes tests/golden/reference_fixtures.npz from the reference's golden
fixtures (tests/data/*.bin of quantumsteve/sunny_gen_eigensolver, produced
there by tests/common/lapack_reference.cpp with LAPACKE_zhegvd).

The 31 MB of fixture inputs are not copied: the oracle's C++ restatement of
the reference generator (oracle/fixture_gen.cpp) regenerates H and S from
(N, B, seed, mode), and this script checks that it does so bit-for-bit
before recording, per fixture, the SHA-256 of H and S (column-major bytes,
as in the file), all eigenvalues W, and the eigenvectors U of the first two
matrices for N in {16, 54}.

Run (needs a checkout of the reference):  python tests/golden/make_golden.py REF_ROOT
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO))
from oracle import fixtures  # noqa: E402

U_SIZES = (16, 54)


def colmajor_bytes(M):
    return np.ascontiguousarray(M.transpose(0, 2, 1)).tobytes()


def main(ref_root: str) -> None:
    data = Path(ref_root) / "tests" / "data"
    out = {}
    names = []
    for path in sorted(data.glob("*.bin")):
        fx = fixtures.read_geig(path)
        mode = "nearid" if "nearid" in path.name else "random"
        H, S = fixtures.generate(fx["n"], fx["batch"], fx["seed"], mode)
        if not (np.array_equal(H, fx["H"]) and np.array_equal(S, fx["S"])):
            raise SystemExit(f"generator does not reproduce {path.name}")
        key = path.stem
        names.append(key)
        out[f"{key}/meta"] = np.array([fx["n"], fx["batch"], fx["seed"], 1 if mode == "nearid" else 0], dtype=np.int64)
        out[f"{key}/sha_H"] = np.frombuffer(hashlib.sha256(colmajor_bytes(fx["H"])).digest(), dtype=np.uint8)
        out[f"{key}/sha_S"] = np.frombuffer(hashlib.sha256(colmajor_bytes(fx["S"])).digest(), dtype=np.uint8)
        out[f"{key}/W"] = fx["W"]
        if fx["n"] in U_SIZES:
            out[f"{key}/U2"] = fx["U"][:2]
        print(f"{path.name}: N={fx['n']} B={fx['batch']} seed={fx['seed']} mode={mode} regenerated bit-exactly")
    out["names"] = np.array(names)
    np.savez_compressed(REPO / "tests" / "golden" / "reference_fixtures.npz", **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py REF_ROOT  (root of a reference checkout)")
    main(sys.argv[1])
