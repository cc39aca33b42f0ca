// sim.js -- drop-in for the reference's src/sim.js (class Sim,
// src/sim.js:29-601) over the CUDA library, through the Node-API addon.
//
// Same constructor, methods, parameter properties and field names, so the
// reference's src/worker.js and test/NAME.mjs scripts run unchanged (the
// loader hook in napi/loader.mjs points their `./sim.js` and `./solid.js`
// imports here).
//
// Fields (sim.phi, sim.rho, sim.ux, ..., sim.f, sim.h, sim.tag) are host
// mirrors in the reference's layout: a getter refreshes its mirror from the
// device at most once per device step (a version counter), and element writes
// such as the dam preset's `sim.phi[i] = p` (src/worker.js:58-69) are found by
// comparing the mirror with the copy taken when it was downloaded, and
// uploaded before the next device call.  Read fields through the property
// (`sim.phi[i]`), not through a reference kept across steps.
import { addon, RigidSphere, SPHERE_F64 } from './solid.js';

export const FIELD = {
  f: 0, f2: 1, h: 2, h2: 3, rho: 4, ux: 5, uy: 6, uz: 7, phi: 8, phiPrev: 9, tag: 10, tagPrev: 11,
  usx: 12, usy: 13, usz: 14, gx: 15, gy: 16, gz: 17, lap: 18, bodyFx: 19, bodyFy: 20, bodyFz: 21,
};
export const STORAGE = { f32: 0, f16: 1, bf16: 2, f64: 3 };
const PARAMS = ['tau', 'tauPhi', 'sigma', 'gravity', 'rhoL', 'rhoG', 'W', 'mobility'];
// phi before h (reduced storage keeps h relative to phi), tags last
const UPLOAD_ORDER = ['phi', 'rho', 'ux', 'uy', 'uz', 'f', 'f2', 'h', 'h2', 'usx', 'usy', 'usz',
  'gx', 'gy', 'gz', 'lap', 'bodyFx', 'bodyFy', 'bodyFz', 'tag', 'tagPrev', 'phiPrev'];
// D3Q27 velocity set, rest first then opposite pairs (src/lattices.js:34-49)
const DIRS = [
  [0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
  [1, 1, 0], [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1], [1, 0, -1],
  [-1, 0, 1], [0, 1, 1], [0, -1, -1], [0, 1, -1], [0, -1, 1], [1, 1, 1], [-1, -1, -1],
  [1, 1, -1], [-1, -1, 1], [1, -1, 1], [-1, 1, -1], [-1, 1, 1], [1, -1, -1],
];

// RigidSpheres behind a solid argument; null for a duck-typed solid of any
// other kind (README.md:69-73), which takes the generic route below
function spheresOf(solid) {
  if (solid == null) return [];
  if (solid instanceof RigidSphere) return [solid];
  if (Array.isArray(solid.spheres) && solid.spheres.every((s) => s instanceof RigidSphere)) return solid.spheres;
  return null;
}

export class Sim {
  constructor(nx, ny, nz, storage = 'f32', device = 0) {
    this.nx = nx; this.ny = ny; this.nz = nz;
    this.n = nx * ny * nz;
    this._h = addon.create(nx, ny, nz, STORAGE[storage] ?? storage, device);
    this._params = new Float64Array(8);
    addon.getParams(this._h, this._params);  // the reference's defaults (src/sim.js:88-95)
    this._paramsDirty = false;
    this._version = 0;
    this._mirrors = new Map();  // field -> { arr, copy, version }
    this._sphereBuf = new Float64Array(SPHERE_F64 * 8);
    this._impulses = new Float64Array(6 * 8);
    // pull offsets (src/sim.js:71-85)
    const nxny = nx * ny;
    this.neighOffset27 = new Int32Array(27);
    this.fOffset27 = new Int32Array(27);
    for (let k = 0; k < 27; k++) {
      const [ex, ey, ez] = DIRS[k];
      this.neighOffset27[k] = -(ez * nxny + ey * nx + ex);
      this.fOffset27[k] = this.neighOffset27[k] * 27 + k;
    }
    this.neighOffset7 = this.neighOffset27.slice(0, 7);
    this.hOffset7 = new Int32Array(7);
    for (let k = 0; k < 7; k++) this.hOffset7[k] = this.neighOffset7[k] * 7 + k;
  }

  dispose() { addon.destroy(this._h); }

  idx(x, y, z) { return (z * this.ny + y) * this.nx + x; }
  rhoFromPhi(p) { return this.rhoG + p * (this.rhoL - this.rhoG); }

  // ---------------------------------------------------------------- mirrors
  _count(name) {
    if (name === 'f' || name === 'f2') return this.n * 27;
    if (name === 'h' || name === 'h2') return this.n * 7;
    return this.n;
  }
  _field(name) {
    let m = this._mirrors.get(name);
    if (!m) {
      const T = name === 'tag' || name === 'tagPrev' ? Uint8Array : Float32Array;
      m = { arr: new T(this._count(name)), copy: null, version: -1 };
      this._mirrors.set(name, m);
    }
    if (m.version !== this._version) {
      addon.downloadField(this._h, FIELD[name], m.arr);
      m.copy = m.arr.slice();
      m.version = this._version;
    }
    return m.arr;
  }
  // has the caller written into this mirror since it was downloaded?
  _written(m) {
    const n = m.arr.byteLength;
    const words = n >> 2;
    const a = new Uint32Array(m.arr.buffer, m.arr.byteOffset, words);
    const b = new Uint32Array(m.copy.buffer, m.copy.byteOffset, words);
    for (let i = 0; i < words; i++) if (a[i] !== b[i]) return true;
    if (words << 2 === n) return false;
    const ta = new Uint8Array(m.arr.buffer, m.arr.byteOffset, n);
    const tb = new Uint8Array(m.copy.buffer, m.copy.byteOffset, n);
    for (let i = words << 2; i < n; i++) if (ta[i] !== tb[i]) return true;
    return false;
  }
  // parameters and host-side field writes to the device, before a device call
  _sync() {
    if (this._paramsDirty) {
      addon.setParams(this._h, this._params);
      this._paramsDirty = false;
    }
    const up = [];
    for (const name of UPLOAD_ORDER) {
      const m = this._mirrors.get(name);
      if (m && m.version === this._version && this._written(m)) up.push(name);
    }
    for (const name of up) {
      const m = this._mirrors.get(name);
      addon.uploadField(this._h, FIELD[name], m.arr);
      m.copy = m.arr.slice();
    }
  }
  _moved() { this._version++; }
  _spheres(list) {
    for (let b = 0; b < list.length; b++) this._sphereBuf.set(list[b].state, b * SPHERE_F64);
    return list.length ? this._sphereBuf.subarray(0, list.length * SPHERE_F64) : null;
  }
  _takeBack(list) {
    for (let b = 0; b < list.length; b++) list[b].state.set(this._sphereBuf.subarray(b * SPHERE_F64, (b + 1) * SPHERE_F64));
  }

  // ---------------------------------------------------------------- the reference's methods
  initFlat(waterlineY) {
    for (const m of this._mirrors.values()) m.version = -1;  // initFlat overwrites every field
    this._sync();
    addon.initFlat(this._h, waterlineY);
    this._moved();
  }
  seedHydrostatic() { this._sync(); addon.seedHydrostatic(this._h); this._moved(); }
  computePhiGradients() { this._sync(); addon.computePhiGradients(this._h); this._moved(); }
  retagCells(solid) {
    const list = spheresOf(solid);
    if (list === null) return this._retagGeneric(solid);
    this._sync();
    addon.retagCells(this._h, this._spheres(list));
    this._moved();
  }

  // ---------------------------------------------------------------- duck-typed solids
  // contains / surfaceVelocity are called here for every interior cell, in the
  // reference's order (src/sim.js:214-244), and uploaded as a mask; after the
  // hydro stream the device returns the momentum-exchange links in scan order
  // and each is applied through solid.applyImpulseAtCell (src/sim.js:517-536).
  _retagGeneric(solid) {
    if (solid.useDevice && typeof solid.worldTriangles === 'function') {
      // a mesh body: voxelised on the device (triangles as 9 numbers each;
      // motion = cx cy cz vx vy vz wx wy wz)
      this._sync();
      addon.retagCellsMesh(this._h, Float64Array.from(solid.worldTriangles()),
        Float64Array.of(solid.cx, solid.cy, solid.cz, solid.vx, solid.vy, solid.vz,
                        solid.wx, solid.wy, solid.wz));
      this._moved();
      return;
    }
    const { nx, ny, nz } = this;
    const mask = this._mask ?? (this._mask = new Uint8Array(this.n));
    const us = this._us ?? (this._us = new Float32Array(3 * this.n));
    mask.fill(0);
    us.fill(0);
    const tmp = [0, 0, 0];
    for (let z = 1; z < nz - 1; z++) {
      for (let y = 1; y < ny - 1; y++) {
        for (let x = 1; x < nx - 1; x++) {
          if (!solid.contains(x, y, z)) continue;
          const i = (z * ny + y) * nx + x;
          mask[i] = 1;
          solid.surfaceVelocity(x, y, z, tmp);
          us[3 * i] = tmp[0]; us[3 * i + 1] = tmp[1]; us[3 * i + 2] = tmp[2];
        }
      }
    }
    this._sync();
    addon.retagCellsMask(this._h, mask, us);
    this._moved();
  }
  _applyLinks(solid) {
    const count = addon.solidLinks(this._h);
    if (count === 0) return;
    const cells = new Int32Array(count), dirs = new Int8Array(count), mom = new Float64Array(count);
    addon.solidLinks(this._h, cells, dirs, mom);
    const { nx } = this, nxny = this.nx * this.ny;
    for (let j = 0; j < count; j++) {
      const [ex, ey, ez] = DIRS[dirs[j]];
      const i = cells[j], z = Math.floor(i / nxny), r = i - z * nxny, y = Math.floor(r / nx), x = r - y * nx;
      const m = mom[j];
      solid.applyImpulseAtCell(x - ex, y - ey, z - ez, -m * ex, -m * ey, -m * ez);
    }
  }
  _stepGeneric(solid) {
    this._retagGeneric(solid);
    this.handleFreshCells(solid);
    this.computePhiGradients();
    this.collidePhase();
    this.streamPhase();
    this.collideHydro();
    this.streamHydroAndMacro(solid);
  }
  handleFreshCells() { this._sync(); addon.handleFreshCells(this._h); this._moved(); }
  collidePhase() { this._sync(); addon.collidePhase(this._h); this._moved(); }
  streamPhase() { this._sync(); addon.streamPhase(this._h); this._moved(); }
  collideHydro() { this._sync(); addon.collideHydro(this._h); this._moved(); }
  _withImpulses(call, solid) {
    const list = spheresOf(solid);
    if (list === null) throw new TypeError('a duck-typed solid keeps its own absorbDeadCells');
    this._sync();
    try {
      call(this._h, this._spheres(list), this._impulses);
    } finally {
      this._moved();
    }
    for (let b = 0; b < list.length; b++) list[b].addImpulse(this._impulses, 6 * b);
  }
  streamHydroAndMacro(solid) {
    if (spheresOf(solid) === null) {
      this._sync();
      try {
        addon.streamHydroAndMacro(this._h, null, this._impulses);
      } finally {
        this._moved();
      }
      this._applyLinks(solid);
      return;
    }
    this._withImpulses(addon.streamHydroAndMacro, solid);
  }
  // src/sim.js:202-210 as one fused device step (phase by phase for a
  // duck-typed solid that is not made of RigidSpheres)
  step(solid) {
    if (spheresOf(solid) === null) return this._stepGeneric(solid);
    this._withImpulses(addon.step, solid);
  }
  _absorbDeadCells(solid) { this._withImpulses(addon.absorbDeadCells, solid); }
  // src/sim.js:586-600 (the second argument is ignored, as in the reference)
  packVolume(out) {
    this._sync();
    addon.packVolume(this._h, out);
    return out;
  }

  // ---------------------------------------------------------------- beyond the reference
  // nsteps worker ticks (src/worker.js:96-100) on the device; the spheres'
  // state comes back into their RigidSphere objects
  runCoupled(solid, nsteps, frameEvery = 0, frames = null) {
    const list = spheresOf(solid);
    if (list === null) throw new TypeError('runCoupled integrates RigidSpheres on the device');
    this._sync();
    const buf = this._spheres(list);
    try {
      addon.runCoupled(this._h, buf, nsteps, frameEvery, frames);
    } finally {
      this._moved();
    }
    this._takeBack(list);
    return frames;
  }
  packVolumeAsync(out) { this._sync(); addon.packVolumeAsync(this._h, out); return out; }
  // step(solid) with packVolume fused into it; `out` holds the frame after waitFrames()
  stepFrame(solid, out) {
    if (spheresOf(solid) === null) {
      this.step(solid);
      return this.packVolumeAsync(out);
    }
    this._withImpulses((h, sp, imp) => addon.stepFrame(h, sp, imp, out), solid);
    return out;
  }
  waitFrames() { addon.waitFrames(this._h); }
  waitFrameSlot() { addon.waitFrameSlot(this._h); }
  field64(name) {
    this._sync();
    const out = new Float64Array(this._count(name));
    addon.downloadFieldF64(this._h, FIELD[name], out);
    return out;
  }
}

for (const [i, name] of PARAMS.entries()) {
  Object.defineProperty(Sim.prototype, name, {
    get() { return this._params[i]; },
    set(v) { this._params[i] = v; this._paramsDirty = true; },
    enumerable: true,
  });
}
for (const name of Object.keys(FIELD)) {
  Object.defineProperty(Sim.prototype, name, {
    get() { return this._field(name); },
    set(v) { this._field(name).set(v); },
    enumerable: true,
  });
}
