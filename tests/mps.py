"""Minimal free-format MPS reader for the reference's own fixture files
(test helper; mirrors read_mps, reference src/utils.jl:34-64: QUADOBJ holds
the lower triangle and Q = Q + Q' - diag(Q))."""
import numpy as np
import scipy.sparse as sp


def read_mps(path):
    rows = {}
    row_type = {}
    obj_row = None
    cols = {}
    A_ent, c_ent, q_ent = [], {}, []
    rhs, rng = {}, {}
    lo, up = {}, {}
    section = None
    with open(path) as f:
        for line in f:
            if not line.strip() or line.startswith("*"):
                continue
            if not line[0].isspace():
                section = line.split()[0]
                continue
            t = line.split()
            if section == "ROWS":
                typ, name = t[0], t[1]
                if typ == "N" and obj_row is None:
                    obj_row = name
                elif typ != "N":
                    row_type[name] = typ
                    rows[name] = len(rows)
            elif section == "COLUMNS":
                if "MARKER" in t:
                    continue
                cname = t[0]
                if cname not in cols:
                    cols[cname] = len(cols)
                for k in range(1, len(t) - 1, 2):
                    r, v = t[k], float(t[k + 1])
                    if r == obj_row:
                        c_ent[cname] = c_ent.get(cname, 0.0) + v
                    elif r in rows:
                        A_ent.append((rows[r], cols[cname], v))
            elif section == "RHS":
                toks = t[1:] if len(t) % 2 == 1 else t
                for k in range(0, len(toks) - 1, 2):
                    if toks[k] in rows:
                        rhs[toks[k]] = float(toks[k + 1])
            elif section == "RANGES":
                toks = t[1:] if len(t) % 2 == 1 else t
                for k in range(0, len(toks) - 1, 2):
                    rng[toks[k]] = float(toks[k + 1])
            elif section == "BOUNDS":
                typ, cname = t[0], t[2]
                v = float(t[3]) if len(t) > 3 else 0.0
                if typ in ("LO", "LI"):
                    lo[cname] = v
                elif typ in ("UP", "UI"):
                    up[cname] = v
                    if v < 0 and cname not in lo:
                        lo[cname] = -np.inf
                elif typ == "FX":
                    lo[cname] = up[cname] = v
                elif typ == "FR":
                    lo[cname], up[cname] = -np.inf, np.inf
                elif typ == "MI":
                    lo[cname] = -np.inf
                elif typ == "PL":
                    up[cname] = np.inf
            elif section in ("QUADOBJ", "QMATRIX"):
                q_ent.append((t[0], t[1], float(t[2])))
    n, m = len(cols), len(rows)
    A = sp.csc_matrix(([e[2] for e in A_ent], ([e[0] for e in A_ent], [e[1] for e in A_ent])), shape=(m, n))
    c = np.zeros(n)
    for k, v in c_ent.items():
        c[cols[k]] = v
    qi = [cols[a] for a, b, v in q_ent]
    qj = [cols[b] for a, b, v in q_ent]
    qv = [v for a, b, v in q_ent]
    Q = sp.csc_matrix((qv, (qi, qj)), shape=(n, n))
    Q = (Q + Q.T - sp.diags(Q.diagonal())).tocsc()
    AL = np.full(m, -np.inf)
    AU = np.full(m, np.inf)
    for r, i in rows.items():
        b = rhs.get(r, 0.0)
        typ = row_type[r]
        if typ == "E":
            AL[i] = AU[i] = b
            if r in rng:
                R = rng[r]
                if R > 0:
                    AU[i] = b + abs(R)
                else:
                    AL[i] = b - abs(R)
        elif typ == "L":
            AU[i] = b
            if r in rng:
                AL[i] = b - abs(rng[r])
        elif typ == "G":
            AL[i] = b
            if r in rng:
                AU[i] = b + abs(rng[r])
    l = np.zeros(n)
    u = np.full(n, np.inf)
    for k, i in cols.items():
        if k in lo:
            l[i] = lo[k]
        if k in up:
            u[i] = up[k]
    return Q, c, A, AL, AU, l, u
