"""Child process for tests/test_loaders.py: every ligand of the reference's data
set through gd_load_complex and through the reference frontend built from its
sources, compared field by field.  Run in its own process because the
reference's .ff parser writes one element past its token arrays
(src/frontend/load.C:1091-1096, :1112-1117: `while (dat3) dat3 >> dat1[dat2++]`),
which is harmless or fatal depending on what else the process holds."""

import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE))


def main() -> int:
    from oracle import oracle as O
    from test_loaders import DATA, _compare, _ours, _ref

    lig = DATA / "astex" / "ligands"
    pdb = DATA / "astex" / "proteins" / "1a07C-1.pdb"
    n = 0
    for sdf in sorted(lig.glob("*.sdf")):
        lid = sdf.stem
        ff = lig / f"{lid}-0.8.ff"
        if not ff.exists():
            continue
        want = _ref(O, lid, sdf, ff, pdb, num_temp=1)
        got = _ours(lid, sdf, ff, pdb, num_temp=1)
        _compare(got, want, ligand_only=True)
        n += 1
    print(f"compared {n}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
