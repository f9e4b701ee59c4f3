// Uses libprr through prr_dropin.hpp the way the reference's scene files use
// its glTF loader: GLTFLoader::load(file, MaterialType::Diffuse) for every
// mesh of a .glb / .gltf, plus an emissive sphere and a camera, then
// Renderer::Render. argv[1]: the glTF file; argv[2]: where the linear
// framebuffer (floats) goes.
#include "prr_dropin.hpp"

#include <fstream>

int main(int argc, char **argv) {
    if (argc < 3)
        return 2;
    const int W = 96, H = 72;
    Scene scene;
    for (MeshTriangle *mesh : GLTFLoader::load(argv[1], MaterialType::Diffuse))
        scene.Add(mesh);
    EmissiveMaterial light;
    light.m_emission = Vector3f(20.0f);
    scene.Add(new Sphere(Vector3f(0.3f, 1.4f, 0.2f), 0.25f, &light));
    scene.camera = Camera::create(Vector3f(0.0f, 2.0f, 2.6f), Vector3f(0, 0, 0),
                                  Vector3f(0, 1, 0), 50.0f, 60.0f);
    scene.camera.init(W, H);
    scene.buildBVH();

    Integrator integrator(scene, 6, 0.8f);
    RenderSettings settings;
    settings.width = W;
    settings.height = H;
    settings.minSPP = settings.maxSPP = 64;
    settings.mode = PRR_RENDER_WAVEFRONT;
    settings.seed = 3;
    Renderer r;
    r.Render(scene, integrator, settings);
    std::ofstream(argv[2], std::ios::binary)
        .write((const char *) r.framebuffer().data(), r.framebuffer().size() * sizeof(float));
    return 0;
}
