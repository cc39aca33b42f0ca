// worker_host.mjs -- runs the reference's src/worker.js unchanged in a Node
// worker thread on the CUDA library, in place of the browser page that
// normally drives it (src/main.js): sends `init` with a grid and preset,
// hands each frame's buffer back (`releaseBuf`) as the renderer does, and
// reports frames per second and the sphere's position.
//
//   node claude-vibe-code-raytracing_b200/napi/worker_host.mjs <reference>/src/worker.js \
//        [--nx 40 --ny 28 --nz 40 --preset drop --frames 200]
import { Worker } from 'node:worker_threads';
import { fileURLToPath } from 'node:url';
import path from 'node:path';

const HERE = path.dirname(fileURLToPath(import.meta.url));
const args = process.argv.slice(2);
const workerPath = path.resolve(args[0] ?? 'src/worker.js');
const opt = (name, dflt) => {
  const i = args.indexOf(`--${name}`);
  return i >= 0 ? args[i + 1] : dflt;
};
const nx = +opt('nx', 40), ny = +opt('ny', 28), nz = +opt('nz', 40);
const frames = +opt('frames', 200);

const worker = new Worker(workerPath, {
  execArgv: ['--import', path.join(HERE, 'register.mjs'), '--import', path.join(HERE, 'browser_globals.mjs')],
});
let got = 0;
const t0 = process.hrtime.bigint();
worker.on('message', (m) => {
  if (m.type !== 'frame') return;
  got++;
  worker.postMessage({ type: 'releaseBuf', buffer: m.vol.buffer }, [m.vol.buffer]);
  if (got === frames) {
    const s = Number(process.hrtime.bigint() - t0) * 1e-9;
    console.log(JSON.stringify({ frames: got, seconds: s, frames_per_s: got / s, solid: m.solid }));
    worker.terminate();
  }
});
worker.on('error', (e) => { console.error(e); process.exitCode = 1; });
worker.postMessage({ type: 'init', nx, ny, nz, substeps: 2, preset: opt('preset', 'drop') });
