"""Decoder of FLOCK v4 R1CS bundles (flavor 2) and BLAKE3 hash-chain bundles
(flavor 3) (bincode 1.3 fixint, little endian).

Field order follows the reference's serde structs: Commitment/PcsParams
(crates/flock-core/src/pcs/commit.rs:34-53,143-147), R1csProofLigerito
(proof.rs:18-23), ZerocheckProof (zerocheck.rs:311-327), LincheckProof
(lincheck.rs:2009-2021), BatchOpeningProofLigerito (pcs.rs:45-48),
LigeritoProof (pcs/ligerito.rs:1022-1048) and header (proof_io.rs:961-995);
the chain bundle (proof_io.rs:144-157) adds hash_kind first, the shift proof
(chain.rs:103-112) after the lincheck and the endpoint bits last.
Used by the tests to compare proofs section by section and to check shapes.
"""
import struct


class Reader:
    def __init__(self, b: bytes):
        self.b, self.i = b, 0

    def take(self, n):
        v = self.b[self.i:self.i + n]
        if len(v) != n:
            raise ValueError("truncated")
        self.i += n
        return v

    def u32(self):
        return struct.unpack("<I", self.take(4))[0]

    def u64(self):
        return struct.unpack("<Q", self.take(8))[0]

    def f(self):
        lo, hi = struct.unpack("<QQ", self.take(16))
        return (lo, hi)

    def h(self):
        return self.take(32)

    def vec(self, fn):
        return [fn() for _ in range(self.u64())]


def parse(data: bytes) -> dict:
    r = Reader(data)
    if r.take(5) != b"FLOCK":
        raise ValueError("bad magic")
    ver, flavor = r.take(1)[0], r.take(1)[0]
    out = {"version": ver, "flavor": flavor}
    if flavor == 3:
        out["hash_kind"] = r.u32()
    out["root"] = r.h()
    out["params"] = (r.u64(), r.u64(), r.u64(), r.u32(), r.u32())
    out["zc_round1_ab"] = r.vec(r.f)
    out["zc_round1_c"] = r.vec(r.f)
    out["zc_rounds"] = r.vec(lambda: (r.f(), r.f()))
    out["zc_finals"] = (r.f(), r.f(), r.f())
    out["lc_rounds"] = r.vec(lambda: (r.f(), r.f()))
    out["lc_z_partial"] = r.vec(r.f)
    if flavor == 3:
        out["shift_rounds"] = r.vec(lambda: (r.f(), r.f()))
        out["shift_g"] = r.f()
    out["s_hat_v"] = r.vec(lambda: r.vec(r.f))
    out["lig_initial_root"] = r.h()

    def opening():
        return (r.vec(lambda: r.vec(r.f)), r.vec(r.h))

    out["lig_initial"] = opening()
    out["lig_roots"] = r.vec(r.h)
    out["lig_levels"] = r.vec(opening)
    out["lig_yr"] = r.vec(r.f)
    out["lig_final"] = opening()
    out["lig_msgs"] = r.vec(lambda: (r.f(), r.f()))
    out["lig_grind_nonces"] = r.vec(r.u64)
    out["lig_ood"] = r.vec(r.f)
    out["lig_fold_nonces"] = r.vec(r.u64)
    if flavor == 3:
        out["cv0_bits"] = bytes(r.vec(lambda: r.take(1)[0]))
        out["cv_last_bits"] = bytes(r.vec(lambda: r.take(1)[0]))
    if r.i != len(data):
        raise ValueError("trailing bytes")
    return out


SECTION_ORDER = ("hash_kind", "root", "params", "zc_round1_ab", "zc_round1_c", "zc_rounds", "zc_finals",
                 "lc_rounds", "lc_z_partial", "shift_rounds", "shift_g", "s_hat_v", "lig_initial_root", "lig_msgs", "lig_fold_nonces", "lig_roots",
                 "lig_ood", "lig_grind_nonces", "lig_initial", "lig_levels", "lig_yr", "lig_final")


def first_difference(a: bytes, b: bytes):
    """Name of the first (transcript-order) section where two bundles differ."""
    pa, pb = parse(a), parse(b)
    for k in SECTION_ORDER + ("cv0_bits", "cv_last_bits"):
        if pa.get(k) != pb.get(k):
            return k
    return None
