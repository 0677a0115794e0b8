// Drop-in Renderer / Denoiser for tracer.js over the wgpt Node-API addon.
//
// The classes keep tracer.js's method names, arguments and call order (Renderer:
// tracer.js:1719-2417, Denoiser: tracer.js:2418-2638) and borrow its scene packing unchanged
// (packDataFromSchema, packSceneData, prepareTextureArray's layer order, HDRTexture.buildHDRCDF,
// Camera.updateRays2); only the device work goes through the addon.  The canvas becomes a
// headless image: `this.canvas` needs only width and height, and readOutput() fills an rgba8
// array (an ImageData's data, for instance) where the reference copies its storage texture to
// the swap chain.
//
//   const { WgptRenderer, WgptDenoiser } = require('./wgpt-renderer.js')(tracerClasses);
//   const r = new WgptRenderer({ width: 1920, height: 1080 });
//   await r.init();
//   await r.setScene(scene);
//   await r.render(256, 64);                 // tiles of 256, 64 progressive samples
//   const rgba = new Uint8ClampedArray(1920 * 1080 * 4);
//   r.readOutput(rgba);

'use strict';

const wgpt = require('./build/Release/wgpt.node');

// tracerClasses: { Renderer, HDRTexture } from tracer.js (the reference's own packing code).
module.exports = function makeWgptClasses(tracerClasses) {
  const { Renderer, HDRTexture } = tracerClasses;

  // override constants 1..11 of shader.wgsl as the addon's flag bits (tracer.js:2067-2080)
  function flagBits(f) {
    return (f.hasSpheres << 0) | (f.hasCubes << 1) | (f.hasPlanes << 2) | (f.hasCylinders << 3) |
      (f.hasTori << 4) | (f.hasMeshes << 5) | (f.hasListMeshes << 6) | (f.hasHeightMaps << 7) |
      (f.hasLights << 8) | (f.hasSkybox << 9) | (f.misSkybox << 10);
  }

  // The resize of every texture to 512 x 512 that prepareTextureArray does with
  // createImageBitmap (tracer.js:1935-1939), as pixels instead of a GPU texture layer.
  function rgbaPixels512(img) {
    const c = new OffscreenCanvas(512, 512);
    const g = c.getContext('2d');
    g.drawImage(img, 0, 0, 512, 512);
    return g.getImageData(0, 0, 512, 512).data;
  }

  class WgptRenderer {
    constructor(canvas, device = 0) {
      this.canvas = canvas;
      this.deviceIndex = device;
      this.ctx = null;
      this.scene = null;
      this.sceneBvh = null;
      this.frame = 0;
      this.currentFlags = {};
      this.section = { x: 0, y: 0, width: 16, height: 16 };
      this.size = { width: canvas.width, height: canvas.height };
      this.uData = new Float32Array(28);
    }

    // init (tracer.js:1733-1770): a CUDA device instead of a WebGPU adapter
    async init() {
      this.ctx = wgpt.create(this.deviceIndex);
    }

    destroy() {
      if (this.ctx) wgpt.destroy(this.ctx);
      this.ctx = null;
    }

    async prepareTextureData(scene) {
      const texs = scene.getTextures();
      if (!texs.length) return null;
      await Promise.all(texs.map((t) => t.loaded));
      const data = new Uint8Array(512 * 512 * 4 * texs.length);
      texs.forEach((t, i) => {
        t.texIndex = i;   // as prepareTextureArray assigns it (tracer.js:1943-1950)
        data.set(rgbaPixels512(t.image), i * 512 * 512 * 4);
      });
      return { data, layers: texs.length };
    }

    sceneDesc(sceneData, sky, cdf, tex) {
      return {
        mat: sceneData.mat.data, object: sceneData.object.data, tlas: sceneData.tlas.data,
        mesh: sceneData.mesh.data, bvh: sceneData.bvh.data, triangle: sceneData.triangle.data,
        plane: sceneData.plane.data, light: sceneData.light.data, skyCDF: cdf.skyCDF,
        sky16: new Uint16Array(sky.data.buffer, sky.data.byteOffset, sky.data.length),
        skyW: sky.width, skyH: sky.height, bounces: this.scene.bounces,
        flags: flagBits(sceneData.flags),
        tex: tex ? tex.data : undefined, texW: 512, texH: 512, texLayers: tex ? tex.layers : 0,
      };
    }

    // setScene (tracer.js:1955-2102): textures, sky, CDF, packing, then one upload
    async setScene(scene, isgbuf = false) {
      this.isgbuf = isgbuf;
      this.scene = scene;
      const tex = await this.prepareTextureData(scene);
      const skybox = scene.background;
      if (!(skybox instanceof HDRTexture)) throw new Error('scene.background must be an HDRTexture');
      await Promise.resolve(skybox.loaded);
      const cdf = skybox.buildHDRCDF();
      this.sceneBvh = null;   // fresh TLAS builder, as setScene does
      const sceneData = this.packSceneData(true);
      this.currentFlags = sceneData.flags;
      wgpt.setScene(this.ctx, this.sceneDesc(sceneData, skybox, cdf, tex));
      this.skyboxData = {
        total_lum: cdf.totalWeight, width: skybox.width, height: skybox.height,
        sky_cdf_index: cdf.sky_cdf_index,
      };
      this.resize();
      this.reset();
    }

    // updateObjects (tracer.js:2132-2164): the five-buffer fast path, setScene otherwise
    async updateObjects() {
      if (!this.scene || !this.ctx) return;
      const sceneData = this.packSceneData(false);
      const flagsMatch = Object.keys(sceneData.flags).every((k) => sceneData.flags[k] === this.currentFlags[k]);
      const fast = flagsMatch && wgpt.updateObjects(this.ctx, {
        mat: sceneData.mat.data, object: sceneData.object.data, tlas: sceneData.tlas.data,
        mesh: sceneData.mesh.data, plane: sceneData.plane.data, flags: flagBits(sceneData.flags),
      });
      if (!fast) {
        console.warn('Buffer capacity or pipeline constants changed. Executing full scene rebuild.');
        await this.setScene(this.scene);
      }
    }

    // resize (tracer.js:2166-2205)
    resize() {
      if (!this.ctx || !this.scene) return;
      wgpt.resize(this.ctx, this.canvas.width, this.canvas.height, !!this.isgbuf);
      this.reset();
    }

    // updateUniforms (tracer.js:2207-2240): the same 28-float block
    updateUniforms() {
      const cam = this.scene.camera;
      cam.updateRays2();
      const randomSeed = Math.floor(Math.random() * 0xFFFFFFFF);
      const uData = this.uData;
      const v = new DataView(uData.buffer);
      uData.set(cam.jitteredPosition, 0);
      v.setUint32(3 * 4, this.frame, true);
      uData.set(cam.ray00, 4);
      v.setUint32(7 * 4, this.size.width, true);
      uData.set(cam.ray10, 8);
      v.setUint32(11 * 4, this.size.height, true);
      uData.set(cam.ray01, 12);
      v.setFloat32(15 * 4, cam.exposure, true);
      uData.set(cam.ray11, 16);
      v.setUint32(19 * 4, randomSeed, true);
      v.setUint32(20 * 4, this.skyboxData.width, true);
      v.setUint32(21 * 4, this.skyboxData.height, true);
      v.setFloat32(22 * 4, this.skyboxData.total_lum, true);
      v.setFloat32(23 * 4, this.totalLightPower, true);
      v.setUint32(24 * 4, this.section.x, true);
      v.setUint32(25 * 4, this.section.y, true);
      v.setUint32(26 * 4, this.skyboxData.sky_cdf_index, true);
      wgpt.setParams(this.ctx, uData);
    }

    // render (tracer.js:2242-2297): tile by tile, `reps` frames per tile, awaiting each tile as
    // the reference awaits onSubmittedWorkDone
    async render(tsize = 256, reps = 1) {
      if (!this.scene) return;
      const { canvas } = this;
      const startingFrame = this.frame;
      const tilesX = Math.ceil(canvas.width / tsize);
      const tilesY = Math.ceil(canvas.height / tsize);
      this.size = { width: canvas.width, height: canvas.height };
      for (let y = 0; y < tilesY; y++) {
        for (let x = 0; x < tilesX; x++) {
          const left = x * tsize;
          const top = y * tsize;
          this.section = {
            x: left, y: top,
            width: Math.min(tsize, canvas.width - left), height: Math.min(tsize, canvas.height - top),
          };
          this.frame = startingFrame;
          await this.renderSection(reps);
        }
      }
      this.frame = startingFrame + reps;
    }

    // renderSection (tracer.js:2299-2309): `reps` frames of one section in one call
    async renderSection(reps = 1) {
      this.updateUniforms();
      const s = this.section;
      if (this.isgbuf) {
        wgpt.renderGBuffer(this.ctx, s.x, s.y, s.width, s.height);
        await wgpt.synchronizeAsync(this.ctx);
      } else {
        await wgpt.renderAsync(this.ctx, this.frame, reps, s.x, s.y, s.width, s.height);
      }
    }

    async initPreview(targetTime) {
      this.targetFrameTime = targetTime || 1000 / 60;
      this.currentPreviewSize = 128;
      this.lastFrameTime = performance.now();
    }

    // renderPreview (tracer.js:2334-2392): adaptive preview size, one frame, scale.wgsl blit
    async renderPreview(canvasRgba8) {
      const { canvas } = this;
      if (this.frame < 16) {
        const now = performance.now();
        const frameTime = now - this.lastFrameTime;
        this.lastFrameTime = now;
        let newPrev = this.currentPreviewSize + (this.targetFrameTime / frameTime - 1.0) * 20;
        newPrev = Math.min(Math.max(canvas.width, canvas.height), Math.max(64, newPrev));
        if (Math.abs(this.currentPreviewSize - newPrev) > 4) {
          this.currentPreviewSize = newPrev;
          this.frame = 0;
        }
      }
      const maxsize = Math.floor(this.currentPreviewSize);
      const scale = Math.min(maxsize / canvas.width, maxsize / canvas.height);
      const pWidth = Math.floor(canvas.width * scale);
      const pHeight = Math.floor(canvas.height * scale);
      this.size = { width: pWidth, height: pHeight };
      this.section = { x: 0, y: 0, width: pWidth, height: pHeight };
      await this.renderSection(1);
      const ratio = new Float32Array([pWidth / canvas.width, pHeight / canvas.height]);
      wgpt.resample(this.ctx, canvas.width, canvas.height, ratio[0], ratio[1]);
      if (canvasRgba8) wgpt.readCanvas(this.ctx, canvasRgba8, canvas.width, canvas.height);
      this.frame++;
    }

    reset() {
      this.frame = 0;
    }

    // SaveRender / the copy to the swap chain: the rgba8 image of the last render or denoise
    readOutput(rgba8) {
      wgpt.readOutput(this.ctx, rgba8);
      return rgba8;
    }

    readAccum(f32) {
      wgpt.readAccum(this.ctx, f32);
      return f32;
    }
  }

  // the reference's packing code, unchanged (tracer.js:1772-1917)
  WgptRenderer.prototype.packDataFromSchema = Renderer.prototype.packDataFromSchema;
  WgptRenderer.prototype.packSceneData = Renderer.prototype.packSceneData;

  class WgptDenoiser {
    // constructor defaults of tracer.js:2419-2447
    constructor(renderer) {
      this.r = renderer;
      this.passes = 4;
      this.sigmaColor = 0.30;
      this.sigmaNormal = 128.0;
      this.sigmaDepth = 0.2;
      this.sigmaAlbedo = 0.07;
      this.sigmaMaterial = 0.07;
      this.glossyProtect = 0.75;
      this.exposure = renderer.scene.camera.exposure;
      this.useMedian = true;
      this.useDemodulate = true;
      this.uBufData = new ArrayBuffer(48);
      // "asRun" reproduces the reference as it runs (every pass reads the last step width,
      // tracer.js:2603-2636); "intended" gives 1, 2, 4, ... as its loop computes
      this.stepMode = 'asRun';
    }

    async init() {}

    setupBuffers() {}

    // updateUniforms (tracer.js:2560-2581)
    updateUniforms() {
      const f32 = new Float32Array(this.uBufData);
      const u32 = new Uint32Array(this.uBufData);
      u32[0] = this.r.canvas.width;
      u32[1] = this.r.canvas.height;
      u32[2] = 1;
      u32[3] = this.passes;
      f32[4] = this.sigmaColor;
      f32[5] = this.sigmaNormal;
      f32[6] = this.sigmaDepth;
      f32[7] = this.sigmaAlbedo;
      f32[8] = this.sigmaMaterial;
      f32[9] = this.glossyProtect;
      f32[10] = this.exposure;
      u32[11] = (this.useMedian ? 1 : 0) | (this.useDemodulate ? 2 : 0);
    }

    // execute (tracer.js:2583-2637): prepass, the a-trous passes and the composite in one call
    execute() {
      this.updateUniforms();
      const steps = new Uint32Array(this.passes);
      for (let i = 0; i < this.passes; i++) steps[i] = this.stepMode === 'asRun' ? 1 << (this.passes - 1) : 1 << i;
      wgpt.denoise(this.r.ctx, new Uint8Array(this.uBufData), steps, this.passes);
    }
  }

  // The learned denoiser: the same call site as Denoiser.execute, with trained weights.
  class WgptLearnedDenoiser {
    constructor(renderer, device = 0, seed = 1) {
      this.r = renderer;
      this.k = wgpt.kpcnCreate(device, seed);
      this.exposure = renderer.scene.camera.exposure;
    }

    loadWeights(float32Params) {
      wgpt.kpcnSetParams(this.k, float32Params);
    }

    execute() {
      wgpt.kpcnDenoise(this.k, this.r.ctx, this.exposure, null);
    }

    destroy() {
      wgpt.kpcnDestroy(this.k);
    }
  }

  return { WgptRenderer, WgptDenoiser, WgptLearnedDenoiser, wgpt };
};
