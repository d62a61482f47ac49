"""Hodgkin-Huxley cable models for the warp-per-system tests (equation strings)."""

def hh_cable(nc):
    """Equations of an nc-compartment Hodgkin-Huxley cable: states V, m, h, n per compartment (grouped by
    variable), parameters gNa, gK, gc, driver I injected into compartment 0, sealed ends."""
    eqs = []
    V = [f"V{j:02d}" for j in range(nc)]
    for j in range(nc):
        v, m, h, n = V[j], f"m{j:02d}", f"h{j:02d}", f"n{j:02d}"
        left = V[j - 1] if j > 0 else v
        right = V[j + 1] if j < nc - 1 else v
        inj = "I + " if j == 0 else ""
        eqs.append(f"d{v} = ({inj}gc * ({left} - 2 * {v} + {right}) - gNa * {m}**3 * {h} * ({v} - 50.0)"
                   f" - gK * {n}**4 * ({v} + 77.0) - 0.3 * ({v} + 54.4)) / 1.0")
    for j in range(nc):
        v, m = V[j], f"m{j:02d}"
        eqs.append(f"d{m} = 0.1 * ({v} + 40.0) / (1 - exp(-({v} + 40.0) / 10.0)) * (1 - {m}) - 4.0 * exp(-({v} + 65.0) / 18.0) * {m}")
    for j in range(nc):
        v, h = V[j], f"h{j:02d}"
        eqs.append(f"d{h} = 0.07 * exp(-({v} + 65.0) / 20.0) * (1 - {h}) - 1.0 / (1 + exp(-({v} + 35.0) / 10.0)) * {h}")
    for j in range(nc):
        v, n = V[j], f"n{j:02d}"
        eqs.append(f"d{n} = 0.01 * ({v} + 55.0) / (1 - exp(-({v} + 55.0) / 10.0)) * (1 - {n}) - 0.125 * exp(-({v} + 65.0) / 80.0) * {n}")
    states = {f"V{j:02d}": -65.0 for j in range(nc)}
    states.update({f"m{j:02d}": 0.05 for j in range(nc)})
    states.update({f"h{j:02d}": 0.6 for j in range(nc)})
    states.update({f"n{j:02d}": 0.32 for j in range(nc)})
    return eqs, states, {"gNa": 120.0, "gK": 36.0, "gc": 0.5}, ["I"]
