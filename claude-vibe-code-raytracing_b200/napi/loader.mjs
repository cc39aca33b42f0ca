// loader.mjs -- Node module hooks that run the reference's own JavaScript
// (src/worker.js, test/NAME.mjs) unchanged on the CUDA library: an import of
// `./sim.js` or `./solid.js` (or `../src/sim.js` ...) from a file outside
// this directory resolves to this directory's sim.js / solid.js, and the
// reference's .js files load as ES modules (they use import/export and ship
// no package.json).  Registered by register.mjs.
import { fileURLToPath, pathToFileURL } from 'node:url';
import path from 'node:path';

const HERE = path.dirname(fileURLToPath(import.meta.url));
const OURS = { 'sim.js': path.join(HERE, 'sim.js'), 'solid.js': path.join(HERE, 'solid.js') };

function outside(url) {
  return url && url.startsWith('file:') && !fileURLToPath(url).startsWith(HERE + path.sep);
}

export async function resolve(specifier, context, nextResolve) {
  const base = path.posix.basename(specifier);
  if ((specifier.startsWith('./') || specifier.startsWith('../')) && OURS[base] && outside(context.parentURL)) {
    return { url: pathToFileURL(OURS[base]).href, shortCircuit: true };
  }
  return nextResolve(specifier, context);
}

export async function load(url, context, nextLoad) {
  if (outside(url) && url.endsWith('.js')) return nextLoad(url, { ...context, format: 'module' });
  return nextLoad(url, context);
}
