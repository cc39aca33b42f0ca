// register.mjs -- `node --import <this file> script` installs loader.mjs.
import { register } from 'node:module';

register('./loader.mjs', import.meta.url);
