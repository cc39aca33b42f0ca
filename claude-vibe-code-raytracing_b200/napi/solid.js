// solid.js -- drop-in for the reference's src/solid.js (class RigidSphere,
// src/solid.js:8-211) whose state lives in the memory the CUDA library reads.
//
// Each sphere keeps its state in a Float64Array of 23 numbers laid out as the
// C ABI's lbm_sphere (include/lbm_b200.h): cx cy cz r vx vy vz wx wy wz
// density mass I dragTargetX dragTargetY dragTargetZ Fx Fy Fz Tx Ty Tz, then
// the int32 `dragging` in the low half of the last element.  Properties read
// and write that array, so sim.step(solid) hands it to the addon without
// copying, and RigidSphere.step runs the library's FP64 integrator
// (lbm_sphere_step_host, the same code as the device-resident loop).
import { createRequire } from 'node:module';

const require = createRequire(import.meta.url);
export const addon = require(process.env.LBM_B200_ADDON ?? './build/lbm_b200.node');

export const SPHERE_F64 = 23;
const SLOT = {
  cx: 0, cy: 1, cz: 2, r: 3, vx: 4, vy: 5, vz: 6, wx: 7, wy: 8, wz: 9,
  density: 10, mass: 11, I: 12, dragTargetX: 13, dragTargetY: 14, dragTargetZ: 15,
  Fx: 16, Fy: 17, Fz: 18, Tx: 19, Ty: 20, Tz: 21,
};

export class RigidSphere {
  constructor(nx, ny, nz, opts = {}) {
    this.nx = nx; this.ny = ny; this.nz = nz;
    this.state = new Float64Array(SPHERE_F64);
    this._flags = new Int32Array(this.state.buffer);  // [44] = dragging
    this.cx = opts.cx ?? nx * 0.5;
    this.cy = opts.cy ?? ny * 0.3;
    this.cz = opts.cz ?? nz * 0.5;
    this.r = opts.r ?? Math.min(nx, ny, nz) * 0.10;
    this.density = opts.density ?? 1.4;
    this.recomputeMass();
  }

  get dragging() { return this._flags[2 * (SPHERE_F64 - 1)] !== 0; }
  set dragging(v) { this._flags[2 * (SPHERE_F64 - 1)] = v ? 1 : 0; }

  // src/solid.js:39-47: volume, mass and moment of inertia of a solid ball
  recomputeMass() {
    const r = this.r;
    this.volume = (4 / 3) * Math.PI * r * r * r;
    this.mass = this.density * this.volume;
    this.I = (2 / 5) * this.mass * r * r;
  }
  setRadius(r) { this.r = r; this.recomputeMass(); }
  setDensity(d) { this.density = d; this.recomputeMass(); }

  // The duck-typed solid interface (README.md:69-73).  The device evaluates
  // the same tests for every cell in FP64; these serve callers that ask the
  // sphere directly.
  contains(x, y, z) {
    const dx = x + 0.5 - this.cx, dy = y + 0.5 - this.cy, dz = z + 0.5 - this.cz;
    return dx * dx + dy * dy + dz * dz <= this.r * this.r;
  }
  surfaceVelocity(x, y, z, out) {
    const rx = x + 0.5 - this.cx, ry = y + 0.5 - this.cy, rz = z + 0.5 - this.cz;
    out[0] = this.vx + (this.wy * rz - this.wz * ry);
    out[1] = this.vy + (this.wz * rx - this.wx * rz);
    out[2] = this.vz + (this.wx * ry - this.wy * rx);
  }
  applyImpulseAtCell(x, y, z, px, py, pz) {
    const rx = x + 0.5 - this.cx, ry = y + 0.5 - this.cy, rz = z + 0.5 - this.cz;
    this.Fx += px; this.Fy += py; this.Fz += pz;
    this.Tx += ry * pz - rz * py;
    this.Ty += rz * px - rx * pz;
    this.Tz += rx * py - ry * px;
  }
  // momentum of the cells the sphere covered this step (src/solid.js:87-101),
  // swept on the device
  absorbDeadCells(sim) { sim._absorbDeadCells(this); }
  // src/solid.js:104-210 in the library's FP64 integrator
  step(dt, gravity) {
    addon.sphereStep(this.state, dt, gravity, this.nx, this.ny, this.nz);
  }
  // the impulses the device summed, added as applyImpulseAtCell would
  addImpulse(out, at = 0) {
    this.Fx += out[at]; this.Fy += out[at + 1]; this.Fz += out[at + 2];
    this.Tx += out[at + 3]; this.Ty += out[at + 4]; this.Tz += out[at + 5];
  }
}

for (const [name, slot] of Object.entries(SLOT)) {
  Object.defineProperty(RigidSphere.prototype, name, {
    get() { return this.state[slot]; },
    set(v) { this.state[slot] = v; },
    enumerable: true,
  });
}
