"""Host-side pieces of the adjoint: parameter lists, model perturbations and
the parameter vector of GreenProblem (no GPU)."""
import numpy as np

from ed_solver_b200 import edk
from ed_solver_b200.autograd import GreenProblem
from ed_solver_b200.model import matsubara, workload


def test_star_params_cover_the_32_parameters_of_the_ns16_model():
    m = workload("c5").model
    p = edk.star_params(m)
    assert len(p) == 32
    kinds = [k for k, _, _, _ in p]
    assert kinds.count(edk.PARAM_EB) == 15 and kinds.count(edk.PARAM_VBC) == 15
    assert kinds.count(edk.PARAM_EC) == 1 and kinds.count(edk.PARAM_U) == 1


def test_perturb_moves_symmetric_entries_together():
    m = workload("c2").model
    q = edk.perturb(m, (edk.PARAM_EB, 0, 2, 2), 0.5)
    d = q.eb - m.eb
    assert d[0, 0, 2] == d[0, 2, 0] == d[1, 0, 2] == d[1, 2, 0] == 0.5
    assert np.count_nonzero(d) == 4
    q = edk.perturb(m, (edk.PARAM_VBC, 3, 1, 0), -0.25)
    d = q.vbc - m.vbc
    assert d[0, 3, 1] == -0.25 and np.count_nonzero(d) == 1
    q = edk.perturb(m, (edk.PARAM_U, 0, 1, 0), 1.0)
    assert (q.u - m.u)[0, 1] == (q.u - m.u)[1, 0] == 1.0
    assert np.array_equal(m.eb, workload("c2").model.eb)        # the input is untouched


def test_green_problem_parameter_vector_round_trip():
    m = workload("c1").model
    prob = GreenProblem(ctx=None, model=m, params=edk.star_params(m), sector=(4, 4), chains=[(0, 0, True)],
                        nitergreen=10, wn=matsubara(50.0, 4))
    th = prob.values()
    assert np.allclose(prob.model_at(th).vbc, m.vbc)
    th2 = th + np.linspace(0.01, 0.16, len(th))
    m2 = prob.model_at(th2)
    prob2 = GreenProblem(ctx=None, model=m2, params=prob.params, sector=(4, 4), chains=[(0, 0, True)],
                         nitergreen=10, wn=prob.wn)
    assert np.allclose(prob2.values(), th2)
    assert np.allclose(m2.eb[1], m2.eb[0])                       # spin-symmetric parameters
