"""``NQS`` facade for the RBM variational-Monte-Carlo path, on the GPU.

Keeps the reference's entry points and their argument meaning
(``QES/NQS/nqs.py``): the constructor with ``s_*`` sampler kwargs
(``:241-591``, defaults ``:1027-1041``), ``sample`` (``:1896-1942``),
``step`` (``:2353-2424`` -> ``NQSSingleStepResult``), ``log_derivative``
(``:2134-2188``), ``get_params`` / ``set_params`` and ``train``
(``:3002-3309``; the loop of ``QES/NQS/src/nqs_train.py:1460-1619``).

One training epoch = sample (persistent sampler kernel) -> theta / tanh for
the samples (forward kernel) -> E_loc (fused local-energy kernel) ->
float64 statistics -> SR solve (structured CG) -> float64 Euler/SGD update.
Only the recognised models (TFIM, XXZ, J1-J2) are accepted as the physics;
an arbitrary local-energy callable raises, there is no fallback path.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Any, List, Optional

import numpy as np
import torch

from . import device as dv
from .hamiltonian import SpinHamiltonian
from .rbm import RBM
from .sampler import VMCSampler
from .tdvp import TDVP


@dataclass
class NQSSingleStepResult:
    loss: Any
    loss_mean: Any
    loss_std: Any
    grad_flat: Any
    params_shapes: List
    params_sizes: List
    params_cpx: List


@dataclass
class NQSTrainStats:
    """Per-epoch history, with the reference's field names (``QES/NQS/src/nqs_train.py:136-148``)."""
    history: List[complex] = field(default_factory=list)
    history_std: List[float] = field(default_factory=list)
    lr_history: List[float] = field(default_factory=list)
    diag_history: List[float] = field(default_factory=list)
    sigma2_history: List[float] = field(default_factory=list)
    rhat_history: List[float] = field(default_factory=list)
    acceptance: List[float] = field(default_factory=list)
    cg_iterations: List[int] = field(default_factory=list)
    timings: List[float] = field(default_factory=list)
    seed: Optional[int] = None
    exact_predictions: Optional[np.ndarray] = None
    exact: Optional[float] = None

    @property
    def last_energy(self):
        return self.history[-1] if self.history else None


@dataclass
class NQSObservable:
    """Local values and statistics of one observable (the fields of the reference's ``NQSObservable``,
    ``QES/NQS/src/nqs_engine.py:231-300``)."""
    values: Any
    mean: Any = None
    std: Optional[float] = None
    variance: Optional[float] = None
    error_of_mean: Optional[float] = None
    min_val: Optional[float] = None
    max_val: Optional[float] = None
    n_samples: int = 0
    observable_name: str = ""
    backend_used: str = "cuda"
    has_stats: bool = True

    def summary(self):
        return {"name": self.observable_name, "expectation": self.mean, "std": self.std, "min": self.min_val,
                "max": self.max_val, "variance": self.variance, "error_of_mean": self.error_of_mean,
                "n_samples": self.n_samples}


class NQS:
    def __init__(self, logansatz="rbm", model: SpinHamiltonian = None, hilbert=None, *, sampler="vmc",
                 batch_size=None, backend="cuda", dtype=np.complex64, param_dtype=None, seed=0, alpha=1.0,
                 nparticles=None, device=None, verbose=False, replica: int = 1, **kwargs):
        if model is None or not isinstance(model, SpinHamiltonian):
            raise TypeError("NQS on the GPU path needs a TransverseFieldIsing / XXZ / J1J2Model instance")
        self._model = model
        self._hilbert = hilbert if hilbert is not None else model.hilbert_space
        ns = self._hilbert.ns
        if isinstance(logansatz, RBM):
            self._net = logansatz
        elif str(logansatz).lower() in ("rbm", "r1"):
            self._net = RBM((ns,), alpha=kwargs.pop("alpha_rbm", alpha), dtype=param_dtype or dtype, seed=seed,
                            init_scale=kwargs.pop("init_scale", 0.01), device=device)
        else:
            raise ValueError(f"ansatz {logansatz!r}: the GPU path implements the RBM")
        if self._net.ns != ns:
            raise ValueError("ansatz size does not match the Hilbert space")
        self._batch_size = batch_size
        self._nparticles = ns if nparticles is None else int(nparticles)
        self._seed = seed
        self._sampler = VMCSampler(
            self._net, (ns,), upd_fun=kwargs.get("s_upd_fun", "LOCAL"), mu=kwargs.get("s_mu", 2.0),
            beta=kwargs.get("s_beta", 1.0), therm_steps=kwargs.get("s_therm_steps", 24),
            sweep_steps=kwargs.get("s_sweep_steps", 48), seed=kwargs.get("s_seed", seed), hilbert=self._hilbert,
            numsamples=kwargs.get("s_numsamples", 192), numchains=kwargs.get("s_numchains", 24),
            initstate=kwargs.get("s_initstate", None), logprob_fact=kwargs.get("s_logprob_fact", 0.5),
            n_particles=self._nparticles, lattice=getattr(model, "lattice", None),
            recompute_every=kwargs.get("s_recompute_every", None),
            # parallel tempering: `replica` slots on a geometric ladder, or an explicit `pt_betas`
            pt_replicas=int(replica) if int(replica) > 1 else None, pt_betas=kwargs.get("pt_betas", None))
        self._lowered = model.lower()
        self._dev_ham = dv.DeviceHamiltonian(self._lowered, self._net.device)
        self._eloc_tables = None
        self._eloc_tables_version = -1
        self._eloc_ws = None
        self._tdvp = None
        self.exact = None

    # ------------------------------------------------------------------ accessors
    @property
    def net(self):
        return self._net

    @property
    def sampler(self):
        return self._sampler

    @property
    def model(self):
        return self._model

    @property
    def hilbert(self):
        return self._hilbert

    def get_params(self, unravel=False):
        return self._net.get_params(unravel=unravel)

    def set_params(self, params):
        self._net.set_params(params)

    @property
    def num_params(self):
        return self._net.n_params

    # ------------------------------------------------------------------ overlaps and entropies
    @staticmethod
    def compute_overlap(nqs_a: "NQS", nqs_b: "NQS", *, num_samples: int = 4096, num_chains=None,
                        operator=None, operator_args=None) -> float:
        """F = |<A|B>|^2 / (<A|A><B|B>) = E_A[psi_B/psi_A] E_B[psi_A/psi_B] (``nqs.py:3819-3903``)."""
        if nqs_a.net.ns != nqs_b.net.ns:
            raise ValueError("NQS instances must have the same number of visible units to compute overlap.")
        if operator is not None:
            raise NotImplementedError("operator insertion is not part of the GPU path")

        def log_mean_ratio(src, other):
            bits, lp_src = src.sampler.sample_bits(num_samples)
            _, _, lp_other = dv.rbm_forward(other.net.flat, other.net.ns, other.net.nh, bits, tanh=False)
            lr = (lp_other.to(torch.complex128) - lp_src.to(torch.complex128))
            return torch.logsumexp(lr, dim=0) - np.log(lr.shape[0])

        lm = log_mean_ratio(nqs_a, nqs_b) + log_mean_ratio(nqs_b, nqs_a)
        return float(torch.exp(lm).real.item())

    @staticmethod
    def compute_renyi2(nqs: "NQS", region=None, *, num_samples=None, num_chains=None, exact_sum=False,
                       return_swap_mean=False, return_error=False, min_swap_value=1e-15):
        """Second Renyi entropy of region A by the two-replica swap estimator
        (``nqs.py:3905-3942`` -> ``nqs_entropy.py:311``): two successive sample batches of the sampler
        paired across different chains,
        Tr rho_A^2 = mean[psi(A1,B0) psi(A0,B1) / (psi(A0,B0) psi(A1,B1))], S2 = -ln Tr rho_A^2."""
        if exact_sum:
            raise NotImplementedError("exact_sum: use the exact wavefunction on the host")
        net = nqs.net
        ns = net.ns
        region = np.arange(ns // 2) if region is None else np.asarray(region, dtype=np.int64).reshape(-1)
        mask = np.zeros(dv.n_words(ns), dtype=np.uint32)
        for i in region:
            mask[i >> 5] |= np.uint32(1) << np.uint32(i & 31)
        mask_d = torch.as_tensor(mask.view(np.int32), device=net.device)
        if num_chains is not None:
            nqs.sampler.set_numchains(num_chains)
        b0, _ = nqs.sampler.sample_bits(num_samples)
        b0 = b0.clone()
        b1, _ = nqs.sampler.sample_bits(num_samples)
        # pair each row of the first batch with the next chain's row of the second batch, so that the two
        # replicas come from different Markov chains (same-chain pairs a sweep apart are correlated and
        # bias Tr rho_A^2 upwards)
        b1 = torch.roll(b1, shifts=1, dims=0).contiguous()
        sa, sb = torch.empty_like(b0), torch.empty_like(b0)
        from . import _lib
        _lib.call("qes_swap_region", int(b0.shape[0]), ns, _lib.ptr(mask_d), _lib.ptr(b0), _lib.ptr(b1),
                  _lib.ptr(sa), _lib.ptr(sb), _lib.stream_ptr())
        lp = lambda b: dv.rbm_forward(net.flat, ns, net.nh, b, tanh=False)[2].to(torch.complex128)
        ratio = torch.exp(lp(sa) + lp(sb) - lp(b0) - lp(b1)).real
        tr = float(ratio.mean().item())
        err = float(ratio.std().item() / np.sqrt(ratio.numel()))
        if return_swap_mean:
            return (tr, err) if return_error else tr
        s2 = -np.log(max(tr, min_swap_value))
        return (s2, err / max(tr, min_swap_value)) if return_error else s2

    # ------------------------------------------------------------------ observables
    def _observable_device(self, op):
        cache = self.__dict__.setdefault("_obs_cache", {})
        ent = cache.get(id(op))
        if ent is None or ent[0] is not op:
            ent = (op, dv.DeviceHamiltonian(op.lower(), self._net.device))
            cache[id(op)] = ent
        return ent[1]

    def local_values(self, op, bits, tanh_theta=None):
        """Local values O_loc(s) = sum_s' conj(<s'|O|s>) psi(s') / psi(s) of a lowered spin operator (the
        local-energy kernel with the operator's own move tables), complex64 per sample."""
        if not isinstance(op, SpinHamiltonian):
            raise TypeError("observables on the GPU path are SpinOperator / model instances (a Python callable "
                            "of the reference's form has no device evaluation here)")
        if op.ns != self._net.ns:
            raise ValueError("observable acts on a different number of sites")
        net = self._net
        if tanh_theta is None:
            _, tanh_theta, _ = dv.rbm_forward(net.flat, net.ns, net.nh, bits, theta=False, tanh=True, logpsi=False)
        h = self._observable_device(op)
        tables = dv.move_tables(net.flat, net.ns, net.nh, h.move_i, h.move_j, h.move_kind, move_major=False)
        return dv.local_energy(net.flat, net.ns, net.nh, bits, tanh_theta, h, tables)

    def compute_observable(self, states=None, ansatze=None, functions=None, names=None, *, params=None,
                           probabilities=None, batch_size=None, num_samples=None, num_chains=None, return_stats=True,
                           return_values=False, args=None, **kwargs):
        """Observables on sampled (or given) configurations (``QES/NQS/nqs.py:1565-1600`` ->
        ``nqs_engine.py:543-660``): local values O_loc(s) on states drawn from |psi|^2 (the NQS sampler
        when ``states`` is None), mean and std weighted by ``probabilities`` when given.  ``functions``
        is one operator or a list (SpinOperator or a model); returns one NQSObservable, a list of them,
        or the value arrays with ``return_values``."""
        if args is not None:
            raise NotImplementedError("observable arguments: build one SpinOperator per argument instead")
        if functions is None or (isinstance(functions, (list, tuple)) and len(functions) == 0):
            raise ValueError("At least one observable function must be provided")
        if params is not None:
            self.set_params(params)
        single = not isinstance(functions, (list, tuple))
        ops = [functions] if single else list(functions)
        net = self._net
        if states is None:
            if num_chains is not None:
                self._sampler.set_numchains(num_chains)
            bits, lp = self._sampler.sample_bits(num_samples)
            if probabilities is None:
                probabilities = self._sampler.sample_probs(lp)
        else:
            bits = net.bits(states)
        _, tn, _ = dv.rbm_forward(net.flat, net.ns, net.nh, bits, theta=False, tanh=True, logpsi=False)
        w = None if probabilities is None else dv.sample_weights(probabilities, int(bits.shape[0]), bits.device)
        out, vals = [], []
        for k, op in enumerate(ops):
            v = self.local_values(op, bits, tn)
            vals.append(v)
            if return_values:
                continue
            st = dv.loss_stats(v, w).cpu().numpy()
            n = int(v.shape[0])
            vr = v.real
            name = names[k] if isinstance(names, (list, tuple)) else (names if isinstance(names, str) else
                                                                     getattr(op, "name", f"O_{k}"))
            out.append(NQSObservable(values=v, mean=complex(st[0], st[1]), std=float(st[3]),
                                     variance=float(st[2]), error_of_mean=float(st[3]) / np.sqrt(max(n, 1)),
                                     min_val=float(vr.min()), max_val=float(vr.max()), n_samples=n,
                                     observable_name=name, has_stats=bool(return_stats)))
        if return_values:
            return vals[0] if single else vals
        return out[0] if single else out

    expectation = compute_observable

    def measure(self, observables, **kwargs):
        """One operator, a list, or a mapping name -> operator (then a dict of results keyed by name);
        ``QES/NQS/nqs.py:1602-1660``."""
        if isinstance(observables, dict):
            names = list(observables.keys())
            res = self.compute_observable(functions=list(observables.values()), names=names, **kwargs)
            return {n: r for n, r in zip(names, res)}
        return self.compute_observable(functions=observables, **kwargs)

    # ------------------------------------------------------------------ checkpoints
    def save_checkpoint(self, directory, step, metadata=None, stats: Optional["NQSTrainStats"] = None):
        """The float64 / complex128 parameter tree and metadata in the reference's checkpoint layout
        (``checkpoint_<step>.npz`` with "/"-flattened keys, JSON metadata beside it)."""
        from .checkpoint import NQSCheckpointManager
        meta = {"model": type(self._model).__name__, "ns": self._net.ns, "nh": self._net.nh,
                "dtype": str(self._net.dtype), "seed": self._seed,
                "sampler": {"numchains": self._sampler.numchains, "numsamples": self._sampler.numsamples,
                            "rule": self._sampler._upd_rule_name}}
        if stats is not None:
            meta["history"] = [complex(h) for h in stats.history]
            meta["history_std"] = list(stats.history_std)
        meta.update(metadata or {})
        return NQSCheckpointManager(directory).save(step, self._net.get_params(), meta)

    def load_checkpoint(self, directory, step=None, filename=None):
        """Load a checkpoint written by this package or by the reference (its npz layout); returns its
        metadata."""
        from .checkpoint import NQSCheckpointManager
        mgr = NQSCheckpointManager(directory)
        if step is None and filename is None:
            step = mgr.latest_step
        tree = mgr.load(step, filename=filename)
        if set(tree) == {"params"}:
            self._net.set_params(tree["params"])
        else:
            self._net.set_params(tree)
        return mgr.load_metadata(step, filename=filename)

    # ------------------------------------------------------------------ evaluation
    def ansatz(self, states):
        return self._net.log_psi(states)

    __call__ = ansatz

    def _tables(self):
        if self._eloc_tables is None or self._eloc_tables_version != self._net.version:
            h = self._dev_ham
            self._eloc_tables = dv.move_tables(self._net.flat, self._net.ns, self._net.nh, h.move_i, h.move_j,
                                               h.move_kind, move_major=False)
            self._eloc_tables_version = self._net.version
        return self._eloc_tables

    def local_energy_bits(self, bits, tanh_theta=None):
        net = self._net
        if tanh_theta is None:
            _, tanh_theta, _ = dv.rbm_forward(net.flat, net.ns, net.nh, bits, theta=False, tanh=True, logpsi=False)
        need = dv.local_energy_workspace(dv.dtype_code(net.flat), net.ns, net.nh, int(bits.shape[0]),
                                         self._dev_ham.n_moves)
        if self._eloc_ws is None or self._eloc_ws.numel() < need:
            self._eloc_ws = torch.empty((max(need, 1),), dtype=torch.uint8, device=net.device)
        return dv.local_energy(net.flat, net.ns, net.nh, bits, tanh_theta, self._dev_ham, self._tables(),
                               self._eloc_ws)

    def local_energy(self, states):
        return self.local_energy_bits(self._net.bits(states))

    def log_derivative(self, states, batch_size=None, params=None, *args, **kwargs):
        if params is not None:
            self.set_params(params)
        O = self._net.log_derivative(states)
        return O, self._net.params_shapes, self._net.params_sizes, self._net.params_cpx

    # ------------------------------------------------------------------ sampling / step
    def sample(self, num_samples=None, num_chains=None, reset=False, *, params=None, **kwargs):
        if reset:
            self._sampler.reset()
        out = self._sampler.sample(parameters=params, num_samples=num_samples, num_chains=num_chains)
        if kwargs.get("states", False):
            return out[1]
        if kwargs.get("last", False):
            return out[0]
        return out

    def step(self, configs=None, configs_ansatze=None, probabilities=None, params=None, **kwargs):
        if params is not None:
            self.set_params(params)
        net = self._net
        if configs is None:
            bits, lp = self._sampler.sample_bits(kwargs.get("num_samples", None))
        else:
            bits = net.bits(configs)
        _, tn, _ = dv.rbm_forward(net.flat, net.ns, net.nh, bits, theta=False, tanh=True, logpsi=False)
        eloc = self.local_energy_bits(bits, tn)
        w = None if probabilities is None else torch.as_tensor(probabilities, dtype=torch.float32,
                                                               device=net.device).reshape(-1)
        st = dv.loss_stats(eloc, w)
        O = dv.log_derivatives(net.flat, net.ns, net.nh, bits, tn)
        mean = torch.complex(st[0], st[1])
        return NQSSingleStepResult(loss=eloc, loss_mean=mean, loss_std=st[3], grad_flat=O,
                                   params_shapes=net.params_shapes, params_sizes=net.params_sizes,
                                   params_cpx=net.params_cpx)

    # ------------------------------------------------------------------ training
    def train(self, n_epochs=300, checkpoint_every=50, load_checkpoint=False, *, checkpoint_step=None,
              reset_weights=False, override=True, background=False, lin_solver="scipy_cg", pre_solver=None,
              ode_solver="Euler", tdvp=None, grad_clip=None, n_batch=128, n_update=None, num_samples=None,
              num_chains=None, num_thermal=None, num_sweep=None, pt_betas=None, phases=None, timing_mode="basic",
              early_stopper=None, optimizer="sgd", lower_states=None, lr_scheduler=None, reg_scheduler=None,
              diag_scheduler=None, lr=1e-2, reg=None, lin_sigma=None, lin_is_gram=True, lin_force_mat=False,
              use_sr=True, use_minsr=False, rhs_prefactor=-1.0, diag_shift=1e-3, save_path=None, reset_stats=True,
              use_pbar=True, exact_predictions=None, exact_method=None, upd_fun=None, update_kwargs=None,
              symmetrize=None, sr_tol=1e-8, sr_maxiter=1000, callback=None, **kwargs) -> NQSTrainStats:
        """The training loop of ``NQSTrainer.train`` (``QES/NQS/src/nqs_train.py:1460-1619``) with the
        signature of ``NQS.train`` (``QES/NQS/nqs.py:3002-3062``).

        Implemented: SR / MinSR / plain gradient with Euler (SGD) updates, the sampler overrides,
        parallel-tempering betas, gradient clipping, learning-rate and diagonal-shift schedules given
        as callables ``f(epoch)`` or ``f(epoch, last_loss)``, checkpoints every ``checkpoint_every``
        epochs under ``save_path`` (and ``load_checkpoint`` / ``checkpoint_step`` to resume from one),
        ``reset_weights``.  ``n_batch`` only chunks the reference's evaluation, which does not change
        its results (the reference's chunking-invariance test); the kernels here need no chunking.
        Every option whose effect is not implemented raises (no silent drop): other ODE integrators or
        optimisers, phase and named schedulers, early stopping, excited states (``lower_states``),
        regularisation, symmetrisation, preconditioners other than ``"jacobi"``, linear solvers other than
        CG, MINRES (``"minres"``, ``"minres_qlp"``) and the formed-matrix Cholesky.
        ``pre_solver="jacobi"`` preconditions the CG by 1 / diag(S + shift); ``lin_force_mat=True`` forms S
        on the tensor cores and solves it by a float64 Cholesky factorisation."""
        unsupported = {
            "ode_solver": ode_solver not in ("Euler", "euler", None),
            "optimizer": optimizer not in ("sgd", "SGD", None),
            "phases": phases is not None, "early_stopper": early_stopper is not None,
            "lower_states": bool(lower_states), "reg_scheduler": reg_scheduler is not None,
            "reg": bool(reg), "lin_sigma": lin_sigma is not None,
            "symmetrize": bool(symmetrize), "update_kwargs": bool(update_kwargs), "n_update": n_update is not None,
            "background": bool(background), "exact_method": exact_method is not None,
            "pre_solver": pre_solver is not None and str(getattr(pre_solver, "name", pre_solver)).lower() not in (
                "identity", "none", "jacobi"),
            "lr_scheduler": lr_scheduler is not None and not callable(lr_scheduler),
            "diag_scheduler": diag_scheduler is not None and not callable(diag_scheduler),
        }
        bad = [k for k, v in unsupported.items() if v] + sorted(kwargs)
        if bad:
            raise NotImplementedError(f"NQS.train: options not implemented on the GPU path: {', '.join(bad)}")
        if upd_fun is not None and str(upd_fun).upper() != self._sampler._upd_rule_name:
            raise ValueError("change the update rule at construction (s_upd_fun)")
        if reset_weights:
            self._net.set_params(RBM((self._net.ns,), n_hidden=self._net.nh, dtype=self._net.dtype, seed=self._net.seed,
                                     init_scale=self._net.init_scale, device=self._net.device).get_params(unravel=True))
        if load_checkpoint:
            if save_path is None:
                raise ValueError("load_checkpoint needs save_path (the checkpoint directory)")
            self.load_checkpoint(save_path, step=checkpoint_step)
        if num_chains is not None:
            self._sampler.set_numchains(num_chains)
        if num_sweep is not None:
            self._sampler._sweep_steps = int(num_sweep)
        if num_thermal is not None:
            self._sampler._therm_steps = int(num_thermal)
        if pt_betas is not None:
            self._sampler.set_pt_betas(pt_betas)
        if tdvp is not None:
            self._tdvp = tdvp
        else:
            self._tdvp = TDVP(use_sr=use_sr, use_minsr=use_minsr, rhs_prefactor=rhs_prefactor, sr_lin_solver=lin_solver,
                              sr_diag_shift=diag_shift, sr_tol=sr_tol, sr_maxiter=sr_maxiter, grad_clip=grad_clip,
                              sr_lin_solver_t="gram" if lin_is_gram else "matvec",
                              sr_form_matrix=bool(lin_force_mat), sr_precond=pre_solver)
        stats = NQSTrainStats(seed=self._seed)
        if exact_predictions is not None:
            stats.exact_predictions = np.atleast_1d(np.asarray(exact_predictions))
            stats.exact = float(np.min(np.real(stats.exact_predictions)))
            self.exact = stats.exact

        def sched(f, epoch, default):
            if f is None:
                return default
            try:
                return float(f(epoch, stats.history[-1] if stats.history else None))
            except TypeError:
                return float(f(epoch))
        for epoch in range(int(n_epochs)):
            lr_e = sched(lr_scheduler, epoch, lr)
            shift_e = sched(diag_scheduler, epoch, diag_shift)
            self._tdvp.set_diag_shift(shift_e)
            t0 = time.perf_counter()
            info = self.train_step(num_samples=num_samples, lr=lr_e)
            torch.cuda.synchronize()
            stats.timings.append(time.perf_counter() - t0)
            stats.history.append(info["mean"])
            stats.history_std.append(info["std"])
            stats.lr_history.append(float(lr_e))
            stats.diag_history.append(float(shift_e))
            stats.sigma2_history.append(info["sigma2"])
            stats.rhat_history.append(info["r_hat"])
            stats.acceptance.append(info["acceptance"])
            stats.cg_iterations.append(info["cg_iterations"])
            if callback is not None:
                callback(epoch, info)
            if save_path is not None and checkpoint_every and (epoch + 1) % int(checkpoint_every) == 0:
                self.save_checkpoint(save_path, epoch + 1, stats=stats)
            if not np.isfinite(np.real(info["mean"])):
                break
        return stats

    def train_step(self, num_samples=None, lr=1e-2, tdvp: Optional[TDVP] = None):
        """One VMC epoch on the GPU; returns host-side statistics of this epoch."""
        tdvp = tdvp or self._tdvp or TDVP(rhs_prefactor=-1.0, sr_maxiter=1000)
        net = self._net
        bits, lp = self._sampler.sample_bits(num_samples)
        probs = self._sampler.sample_probs(lp)                  # None when the sampler draws |psi|^2
        _, tn, _ = dv.rbm_forward_step(net.flat, net.ns, net.nh, bits, theta=False, tanh=True, logpsi=False)
        eloc = self.local_energy_bits(bits, tn)
        st = dv.loss_stats(eloc, probs)
        rh = dv.loss_rhat(eloc, self._sampler.numchains)
        x = tdvp.solve(net, bits, tn, eloc, probs=probs)
        dv.param_update(net.flat, net.master, x, lr)
        net.bump()
        s = st.cpu().numpy()
        r = rh.cpu().numpy()
        acc = self._sampler.accepted_ratio.mean().item()
        return {"mean": complex(s[0], s[1]), "var": float(s[2]), "std": float(s[3]), "acceptance": acc,
                "r_hat": float(r[0]), "sigma2": float(r[1]),
                "cg_iterations": int(tdvp.last_info.get("iterations", 0)),
                "cg_converged": bool(tdvp.last_info.get("converged", True))}
