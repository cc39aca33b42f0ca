// browser_globals.mjs -- the Web Worker globals src/worker.js uses (self,
// self.onmessage, postMessage with a transfer list), provided inside a Node
// worker_threads worker.  Imported (--import) before worker.js.
import { parentPort } from 'node:worker_threads';

if (parentPort) {
  globalThis.self = globalThis;
  globalThis.postMessage = (msg, transfer) => parentPort.postMessage(msg, transfer ?? []);
  parentPort.on('message', (data) => {
    if (typeof globalThis.self.onmessage === 'function') globalThis.self.onmessage({ data });
  });
}
