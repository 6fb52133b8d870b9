"""The time step around the velocity solve: run_ice_dynamics_pc with DIVA dynamics.

``PCTimeStepper`` mirrors the predictor/corrector scheme of IMAU-ICE
(ice_dynamics_module.f90:243-432, Robinson et al. 2020) for
``choice_ice_dynamics = 'DIVA'`` and ``choice_timestepping = 'pc'``: the
time-step control (dt_crit_ice from the advective limit and the truncation
error, pc_zeta, pc_eta, the DIVA event clock) is host arithmetic on scalars,
exactly as in the reference, and every field operation is a call of the
context (``pc_predictor``, ``solve_DIVA``, ``pc_corrector``, ``pc_finish``),
so the geometry stays resident on the device between steps.

The ice-dynamics event and, with ``thermo=True``, the thermodynamics event
(run_thermo_model every step, the heat equation every dt_thermo) drive the clock;
climate, SMB/BMB models, GIA, output and calving are outside the velocity path
(SMB_a, BMB_a, T_surf_annual_a and GHF_a are input fields), and the start-up scaling of the linear-solver
tolerances (r_solver_acc, :279-290) has no counterpart because the velocity
solver takes its tolerances from the configuration.
"""


class PCTimeStepper:
    """Region state of the predictor/corrector time stepping (IMAU_ICE_main_model.f90:
    478-545 and ice_dynamics_module.f90:987-996 for the initial values)."""

    def __init__(self, ctx, start_time, end_time, dt_min=0.01, dt_max=10.0, dt_startup_phase=10.0,
                 pc_epsilon=0.5, pc_k_I=0.2, pc_k_p=0.2, pc_eta_min=1e-8, thermo=False, retreat_frames=None):
        self.ctx = ctx
        self.start_time, self.end_time = float(start_time), float(end_time)
        self.dt_min, self.dt_max, self.dt_startup_phase = float(dt_min), float(dt_max), float(dt_startup_phase)
        self.pc_epsilon, self.pc_k_I, self.pc_k_p, self.pc_eta_min = pc_epsilon, pc_k_I, pc_k_p, pc_eta_min
        self.time = self.start_time
        self.dt = self.dt_min
        self.dt_crit_ice = self.dt_min
        self.dt_crit_ice_prev = self.dt_min
        self.t_last_DIVA = self.start_time
        self.t_next_DIVA = self.start_time
        self.pc_zeta = 1.0
        self.pc_eta = pc_epsilon
        self.pc_eta_prev = pc_epsilon
        self.reports = []
        # the thermodynamics event (IMAU_ICE_main_model.f90:545; dt_thermo of the context)
        self.thermo = thermo
        self.dt_thermo = float(ctx.cfg.dt_thermo)
        self.t_next_thermo = self.start_time + self.dt_thermo
        self.do_thermo = False
        self.thermo_solves = 0
        # do_apply_prescribed_retreat_mask: the times (t0, t1) of the two mask frames the
        # caller has uploaded (it replaces them and this pair as the model time moves on)
        self.retreat_frames = retreat_frames

    def _dt_max_now(self):
        """The start-up / wind-down cap of the time step (ice_dynamics_module.f90:292-299)."""
        if self.time <= self.start_time + self.dt_startup_phase:
            return self.dt_min + (self.dt_max - self.dt_min) * ((self.time - self.start_time) / self.dt_startup_phase) ** 2
        if self.time >= self.end_time - self.dt_startup_phase:
            return self.dt_min + (self.dt_max - self.dt_min) * ((self.end_time - self.time) / self.dt_startup_phase) ** 2
        return self.dt_max

    def run_ice_dynamics_pc(self, t_end):
        """One call of run_ice_dynamics_pc (:243-432): when the DIVA event is due, choose
        dt_crit_ice, predict the geometry, solve the velocities on it, correct, and
        estimate the truncation error; then the next step length and Hi_tplusdt_a
        (determine_timesteps_and_actions, :817-941, with the DIVA event only)."""
        ctx = self.ctx
        dt_max = self._dt_max_now()
        if self.time == self.t_next_DIVA:
            dt_crit_adv = ctx.calc_critical_timestep_adv(self.dt_max)
            self.dt_crit_ice_prev = self.dt_crit_ice
            dt_from_pc = ((self.pc_epsilon / self.pc_eta) ** (self.pc_k_I + self.pc_k_p)
                          * (self.pc_epsilon / self.pc_eta_prev) ** (-self.pc_k_p) * self.dt)
            self.dt_crit_ice = max(self.dt_min, max(0.5 * self.dt_crit_ice_prev,
                                                    min(self.dt_max, 2.0 * self.dt_crit_ice_prev, dt_crit_adv,
                                                        dt_from_pc)))
            self.dt_crit_ice = max(self.dt_min, min(dt_max, self.dt_crit_ice))
            self.pc_zeta = self.dt_crit_ice / self.dt_crit_ice_prev
            ctx.pc_predictor(self.dt_crit_ice, self.pc_zeta)
            self.reports.append(ctx.solve_DIVA())
            self.t_last_DIVA = self.time
            self.t_next_DIVA = self.time + self.dt_crit_ice
            self.pc_eta_prev = self.pc_eta
            self.pc_eta = ctx.pc_corrector(self.dt_crit_ice, self.pc_zeta, self.pc_eta_min)
        t_next = min(t_end, self.time + self.dt_max, self.t_next_DIVA)
        if self.thermo:
            self.do_thermo = self.time == self.t_next_thermo
            if self.do_thermo:
                self.t_next_thermo = self.time + self.dt_thermo
            t_next = min(t_next, self.t_next_thermo)
        self.dt = t_next - self.time

    def step(self, t_end=None):
        """One model time step: run_ice_dynamics_pc, [run_thermo_model, solving the heat
        equation when its event is due], then the thickness update at the end of the step
        (update_ice_thickness) and the clock (IMAU_ICE_main_model.f90:117-207)."""
        t_end = self.end_time if t_end is None else t_end
        self.run_ice_dynamics_pc(t_end)
        if self.thermo:
            self.ctx.run_thermo_model(self.do_thermo)
            self.thermo_solves += int(self.do_thermo)
        self.ctx.pc_finish(self.dt)
        if self.retreat_frames is not None:            # the end of update_ice_thickness (:637-640)
            self.ctx.apply_prescribed_retreat_mask(self.time, *self.retreat_frames)
        self.time = self.time + self.dt
        return self.dt

    def run(self, t_end=None, max_steps=None):
        """Steps until t_end (or max_steps); returns the number of steps taken."""
        t_end = self.end_time if t_end is None else t_end
        n = 0
        while self.time < t_end and (max_steps is None or n < max_steps):
            self.step(t_end)
            n += 1
        return n


class DirectTimeStepper:
    """The direct time stepping of SIA, SSA and SIA/SSA dynamics (run_ice_dynamics_direct,
    ice_dynamics_module.f90:63-242, with the dynamics events of
    determine_timesteps_and_actions :817-941): each velocity solve when its event is due,
    its critical time step (calc_critical_timestep_SIA for SIA, _adv for SSA) bounded by
    dt_min and the start-up / wind-down cap, then calc_dHi_dt over the step and the
    thickness update at its end (update_ice_thickness).  The reference refuses DIVA here;
    so does this class."""

    def __init__(self, ctx, start_time, end_time, dt_min=0.01, dt_max=10.0, dt_startup_phase=10.0, thermo=False):
        dyn = _abi_name(ctx, "choice_ice_dynamics")
        if dyn not in ("SIA", "SSA", "SIA/SSA"):
            raise ValueError(f'"direct" time stepping works only with SIA, SSA or SIA/SSA dynamics, not {dyn}')
        self.ctx, self.dyn = ctx, dyn
        self.start_time, self.end_time = float(start_time), float(end_time)
        self.dt_min, self.dt_max, self.dt_startup_phase = float(dt_min), float(dt_max), float(dt_startup_phase)
        self.time = self.start_time
        self.t_next_SIA = self.t_next_SSA = self.start_time
        self.dt_crit_SIA = self.dt_crit_SSA = self.dt_min
        self.dt = 0.0
        self.reports = []
        self.thermo = thermo                     # the thermodynamics event, as in PCTimeStepper
        self.dt_thermo = float(ctx.cfg.dt_thermo)
        self.t_next_thermo = self.start_time + self.dt_thermo
        self.do_thermo = False
        self.thermo_solves = 0

    _dt_max_now = PCTimeStepper._dt_max_now

    def run_ice_dynamics_direct(self, t_end):
        ctx, dt_max = self.ctx, self._dt_max_now()
        if self.dyn in ("SIA", "SIA/SSA") and self.time == self.t_next_SIA:
            self.reports.append(ctx.solve_SIA())
            self.dt_crit_SIA = max(self.dt_min, min(dt_max, ctx.calc_critical_timestep_SIA(self.dt_max)))
            self.t_next_SIA = self.time + self.dt_crit_SIA
        if self.dyn in ("SSA", "SIA/SSA") and self.time == self.t_next_SSA:
            self.reports.append(ctx.solve_SSA())
            self.dt_crit_SSA = max(self.dt_min, min(dt_max, ctx.calc_critical_timestep_adv(self.dt_max)))
            self.t_next_SSA = self.time + self.dt_crit_SSA
        t_next = min(t_end, self.time + self.dt_max)
        if self.dyn in ("SIA", "SIA/SSA"):
            t_next = min(t_next, self.t_next_SIA)
        if self.dyn in ("SSA", "SIA/SSA"):
            t_next = min(t_next, self.t_next_SSA)
        if self.thermo:
            self.do_thermo = self.time == self.t_next_thermo
            if self.do_thermo:
                self.t_next_thermo = self.time + self.dt_thermo
            t_next = min(t_next, self.t_next_thermo)
        self.dt = t_next - self.time
        ctx.calc_dHi_dt(self.dt)

    def step(self, t_end=None):
        """One model time step: run_ice_dynamics_direct, [run_thermo_model], then the
        thickness update at the end of the step (IMAU_ICE_main_model.f90:117-207)."""
        t_end = self.end_time if t_end is None else t_end
        self.run_ice_dynamics_direct(t_end)
        if self.thermo:
            self.ctx.run_thermo_model(self.do_thermo)
            self.thermo_solves += int(self.do_thermo)
        self.ctx.pc_finish(self.dt)
        self.time = self.time + self.dt
        return self.dt


def _abi_name(ctx, field):
    """The configuration's choice as its reference name."""
    from . import _abi
    value = getattr(ctx.cfg, field)
    return {v: k for k, v in _abi.ENUM_OPTIONS[field].items()}.get(value, value)
