"""The main integration loop of a run (main.cpp:113-150) for any stepper
with the MeshBlock interface: new_dt() (the CFL step of the current state)
and step(dt) (one RK3 step) -- a MeshBlock, a Mesh, or the oracle's block.

    t, cycles = evolve(MeshBlock(problem), tlim=1080.0,
                       outputs=[NetcdfOutput("robert", dt=180.0)])

Every cycle takes the CFL step of the current state, the last one cut so
that the run ends at tlim (Mesh::NewTimeStep); the outputs are written at
the start, after every cycle whose time reaches their next output time,
and once more at tlim (Outputs::MakeOutputs, main.cpp:94-95, 137-140 and
the final call after the loop).
"""


def evolve(stepper, tlim, outputs=(), time=0.0, nlim=-1, dt_of=None):
    """Run from `time` to `tlim` (or nlim cycles); returns (time, cycles).
    dt_of(stepper): the CFL step when the stepper has no new_dt()."""
    new_dt = dt_of or (lambda s: s.new_dt())
    for o in outputs:
        o.write(stepper, time)
    ncycle = 0
    dt = new_dt(stepper)
    while time < tlim and (nlim < 0 or ncycle < nlim):
        if tlim - time < dt:
            dt = tlim - time
        stepper.step(dt)
        ncycle += 1
        time += dt
        dt = new_dt(stepper)
        if time < tlim:
            for o in outputs:
                if o.due(time, tlim):
                    o.write(stepper, time)
    for o in outputs:
        if o.due(time, tlim):
            o.write(stepper, time)
    return time, ncycle
