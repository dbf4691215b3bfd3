"""Isotherm-point observables from the production averages <N>, <E>, <EN>, <N^2>, <E^2>.

Restates the reference's host formulas (utility_pack.f:2280-2316) and adds the pooling of
independent chains that replaces the reference's MPI replicas on one GPU."""
import numpy as np

RGAS = 8.314472 / 4184.0  # kcal/mol/K (utility_pack.f:77-113)
KBOLTZ = 1.9872041e-3  # kcal/mol/K


def qst(N, E, EN, N2, temp):
    """Isosteric heat of adsorption (kcal/mol), calc_Qst (utility_pack.f:2280-2290)."""
    return -1.0 * (EN - E * N) / (N2 - N * N) + RGAS * temp


def cv(N, E, EN, N2, E2, temp):
    """Constant-volume heat capacity (kcal/mol/K), calc_Cv (utility_pack.f:2305-2316)."""
    return (3.0 / 2.0 * RGAS) + (E2 - (E * E) - (EN - E * N) ** 2 / (N2 - N * N)) / (N * KBOLTZ * temp * temp)


def pooled(states, temp, species=0):
    """Observables of independent chains of one isotherm point with equal production counts.

    `states`: dicts with N, E, EN, N2, E2 (Batch.state / Server.poll).  The pooled moments are
    the chain means; standard errors come from the spread over chains (jackknife for Q_st and
    Cv)."""
    sfx = "" if species == 0 else f"_{species}"
    m = np.array([[s["N" + sfx], s["E" + sfx], s["EN" + sfx], s["N2" + sfx], s["E2" + sfx]] for s in states], dtype=float)
    n = len(m)
    avg = m.mean(0)
    out = {"N": avg[0], "E": avg[1], "EN": avg[2], "N2": avg[3], "E2": avg[4], "chains": n,
           "Qst": qst(avg[0], avg[1], avg[2], avg[3], temp),
           "Cv": cv(avg[0], avg[1], avg[2], avg[3], avg[4], temp)}
    if n > 1:
        out["N_err"] = m[:, 0].std(ddof=1) / np.sqrt(n)
        out["E_err"] = m[:, 1].std(ddof=1) / np.sqrt(n)
        loo = (avg * n - m) / (n - 1)  # leave-one-out means
        jq = qst(loo[:, 0], loo[:, 1], loo[:, 2], loo[:, 3], temp)
        jc = cv(loo[:, 0], loo[:, 1], loo[:, 2], loo[:, 3], loo[:, 4], temp)
        out["Qst_err"] = float(np.sqrt((n - 1) / n * np.sum((jq - jq.mean()) ** 2)))
        out["Cv_err"] = float(np.sqrt((n - 1) / n * np.sum((jc - jc.mean()) ** 2)))
    return out
