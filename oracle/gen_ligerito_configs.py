"""Extract the reference's Ligerito "fast" ladder configs as C++ initializer data.

The reference embeds configs/ligerito/m{22..35}_fast.toml into its prover and
verifier (crates/flock-core/src/pcs/ligerito.rs:256-345, parse :963-1013).
They are fixed protocol data, so they are carried over verbatim as data: one
row per level with {log_inv_rate, k_recursive, queries, grinding_bits,
fold_grinding_bits, ood_samples} plus the final yr_log_n.

Usage: python gen_ligerito_configs.py REFERENCE_ROOT OUT_INC
Only needed when the reference checkout is present; the generated .inc files
are committed.
"""
import sys
import tomllib
from pathlib import Path


def main() -> None:
    ref, out = Path(sys.argv[1]), Path(sys.argv[2])
    lines = ["// Generated by gen_ligerito_configs.py from the reference's",
             "// configs/ligerito/m*_fast.toml (protocol data carried verbatim).",
             "// {m, {{log_inv_rate, k_recursive, queries, grinding_bits,",
             "//       fold_grinding_bits, ood_samples}, ...}, yr_log_n}"]
    for m in range(22, 36):
        p = ref / "crates/flock-core/configs/ligerito" / f"m{m}_fast.toml"
        cfg = tomllib.loads(p.read_text())
        assert cfg["m"] == m and cfg["initial_k"] == 6
        rows = []
        for lv in cfg["levels"]:
            rows.append("{%d, %d, %d, %d, %d, %d}" % (
                lv["log_inv_rate"], lv["k_recursive"], lv["queries"], lv["grinding_bits"],
                lv.get("fold_grinding_bits", 0), lv.get("ood_samples", 0)))
        lines.append("{%d, {{%s}, %d}}," % (m, ", ".join(rows), cfg["final_block"]["yr_log_n"]))
    out.write_text("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
