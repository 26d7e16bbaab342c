"""Reading the reference's INI decks in the tests: Boost's INI rules (see
mhd2d-solver_b200/plugin/boost_shim) and the reference's defaults for the
keys of its shock-tube and plasma-sheet setups (file_access.cpp:300-395,
614-919), turned into the parameter lists of the device problem generators
(MHD_PROBLEM_SHOCK_TUBE, MHD_PROBLEM_SHEET_LOBES)."""
import re

STATE_KEYS = ("rho", "u", "v", "w", "Bx", "By", "Bz", "p")
BC_NAMES = {"periodic": 1, "dirichlet": 2, "neumann": 3, "open": 4}


def read_ini(path):
    tree, section = {}, None
    with open(path) as f:
        for ln in f:
            ln = ln.strip()
            if not ln or ln[0] in "#;":
                continue
            m = re.match(r"\[(.*)\]", ln)
            if m:
                section = m.group(1).strip()
                tree.setdefault(section, {})
                continue
            key, _, val = ln.partition("=")
            tree.setdefault(section, {})[key.strip()] = val.strip()
    return tree


def _num(tree, key, default):
    try:
        return float(tree.get("problem", {})[key])
    except (KeyError, ValueError):
        return default


def _state(tree, suffix, defaults):
    return [_num(tree, f"{k}_{suffix}", d) for k, d in zip(STATE_KEYS, defaults)]


def problem_of(path):
    """(kind, params, nx, ny, dx, dy, gamma, bc) of a shock-tube or
    plasma-sheet deck; bc in the order left, right, bottom, top."""
    t = read_ini(path)
    pr = t.get("problem", {})
    nx, ny = int(pr.get("Nx", 16)), int(pr.get("Ny", 16))
    gamma = _num(t, "gamma", 1.4)
    bc = tuple(BC_NAMES[pr.get(f"boundary {s}", "open")] for s in ("left", "right", "bottom",
                                                                    "top"))
    kind = pr.get("type")
    if kind == "shock tube":
        lx, ly = _num(t, "Lx", 2.0), _num(t, "Ly", 2.0)
        params = [lx, ly, _num(t, "interface angle", 0.0)]
        params += _state(t, "l", (1.0, 0.0, 0.0, 0.0, 0.75, 1.0, 0.0, 1.0))
        params += _state(t, "r", (0.125, 0.0, 0.0, 0.0, 0.75, -1.0, 0.0, 0.1))
        return "shock tube", params, nx, ny, lx / nx, ly / ny, gamma, bc
    if kind == "plasma sheet":
        lx, ly = _num(t, "Lx", 2.0), _num(t, "Ly", 2.0)
        x0, y0 = _num(t, "start_x", 0.0), _num(t, "start_y", 0.0)
        head = _num(t, "sheet start", x0 + lx / 2)
        foot = _num(t, "sheet start foot", head)
        thick = _num(t, "sheet thickness", ly / 2.0)
        profile = pr.get("sheet profile", "constant")
        trans = pr.get("transition type", "jump")
        points = int(pr.get("transition points", 1))
        params = [lx, ly, x0, y0, head, foot, thick, 1.0 if profile == "tanh" else 0.0,
                  0.0 if trans == "jump" else 1.0, float(points)]
        params += _state(t, "l", (0.1, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.1))
        params += _state(t, "r", (1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0))
        params += _state(t, "u", (0.1, 0.0, 0.0, 0.0, -0.5, 0.0, 0.0, 0.875))
        params += _state(t, "d", (0.1, 0.0, 0.0, 0.0, 0.5, 0.0, 0.0, 0.875))
        return "plasma sheet", params, nx, ny, lx / nx, ly / ny, gamma, bc
    raise ValueError(f"{path}: problem type {kind!r} has no device generator here")
