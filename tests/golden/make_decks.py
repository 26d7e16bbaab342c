"""Write the reduced INI decks under tests/golden/decks/ from the reference's
own example decks (example-inputs/*.ini of the reference checkout).

Each deck keeps the reference's text and changes only the keys listed
below: smaller grids and end times (so both the reference program and the
drop-in program finish in seconds), full-precision binary grid dumps (the
example decks write floats, which would hide differences below 1e-7), and
for some decks another scheme, time method or characteristics logging, so
that every plugin class runs.

Usage:  python tests/golden/make_decks.py [reference checkout]
        (default: $MHD2D_REFERENCE, else /root/reference)
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "decks")

# output name -> (example deck, {(section, key): value})
DOUBLE = {("output grid", "binary use double"): "true"}
DECKS = {
    "bw_lf": ("bw-shock-tube.ini", {("time", "t_max"): "0.1", **DOUBLE}),
    "bw_roe_chars": ("bw-shock-tube.ini", {("problem", "space method"): "eno-roe",
                                           ("time", "t_max"): "0.1",
                                           ("logging", "characteristics"): "true", **DOUBLE}),
    "explosion_lf": ("explosion.ini", {("problem", "Nx"): "32", ("problem", "Ny"): "32",
                                       ("time", "t_max"): "0.05", **DOUBLE}),
    "ot_lf_float": ("ot-vortex.ini", {("problem", "Nx"): "32", ("problem", "Ny"): "32",
                                      ("time", "t_max"): "0.1"}),
    "ot_roe_euler": ("ot-vortex.ini", {("problem", "Nx"): "32", ("problem", "Ny"): "24",
                                       ("problem", "space method"): "eno-roe",
                                       ("problem", "time method"): "euler",
                                       ("time", "t_max"): "0.05", **DOUBLE}),
    "ot_central": ("ot-vortex.ini", {("problem", "Nx"): "32", ("problem", "Ny"): "32",
                                     ("problem", "space method"): "central fd",
                                     ("time", "t_max"): "0.05", **DOUBLE}),
    "sheet_lf": ("plasma-sheet.ini", {("problem", "Nx"): "64", ("problem", "Ny"): "12",
                                      ("time", "t_max"): "0.1", **DOUBLE}),
    "wave_alfven_lf": ("wave-test-2-neg-alfven.ini", {("problem", "Nx"): "32",
                                                      ("problem", "Ny"): "32",
                                                      ("time", "t_max"): "0.1", **DOUBLE}),
    "wave_fast_roe": ("wave-test-7-pos-fast-ms.ini", {("problem", "Nx"): "32",
                                                      ("problem", "Ny"): "16",
                                                      ("problem", "space method"): "eno-roe",
                                                      ("time", "t_max"): "0.1", **DOUBLE}),
}


def rewrite(text, changes):
    """The deck's lines with the listed keys of the listed sections replaced
    (keys that the deck lacks are added at the end of their section)."""
    out, section, seen = [], None, set()
    lines = text.splitlines()

    def flush(sec):
        for (s, k), v in changes.items():
            if s == sec and (s, k) not in seen:
                out.append(f"{k} = {v}")
                seen.add((s, k))

    for ln in lines:
        m = re.match(r"\s*\[(.+)\]\s*$", ln)
        if m:
            flush(section)
            section = m.group(1).strip()
            out.append(ln)
            continue
        kv = re.match(r"\s*([^#;=][^=]*?)\s*=", ln)
        if kv and (section, kv.group(1)) in changes:
            key = kv.group(1)
            out.append(f"{key} = {changes[(section, key)]}")
            seen.add((section, key))
            continue
        out.append(ln)
    flush(section)
    missing = set(changes) - seen
    if missing:
        raise ValueError(f"sections missing for {sorted(missing)}")
    return "\n".join(out) + "\n"


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MHD2D_REFERENCE",
                                                               "/root/reference")
    src = os.path.join(ref, "example-inputs")
    os.makedirs(OUT, exist_ok=True)
    for name, (deck, changes) in DECKS.items():
        with open(os.path.join(src, deck)) as f:
            text = f.read()
        with open(os.path.join(OUT, name + ".ini"), "w") as f:
            f.write(rewrite(text, changes))
    print(f"wrote {len(DECKS)} decks to {OUT}")


if __name__ == "__main__":
    main()
