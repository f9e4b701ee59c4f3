// Uses libprr through prr_dropin.hpp the way the reference's scene code uses
// its OBJ constructor: MeshTriangle(filename, offset, material), plus an
// emissive sphere and a camera, then Renderer::Render. argv[1]: the .obj file;
// argv[2]: where the linear framebuffer (floats) goes.
#include "prr_dropin.hpp"

#include <fstream>

int main(int argc, char **argv) {
    if (argc < 3)
        return 2;
    const int W = 80, H = 60;
    Scene scene;
    DiffuseMaterial grey;
    grey.baseColor = Vector3f(0.7f, 0.6f, 0.5f);
    scene.Add(new MeshTriangle(argv[1], Vector3f(-0.5f, 0.0f, -0.5f), &grey));
    EmissiveMaterial light;
    light.m_emission = Vector3f(15.0f);
    scene.Add(new Sphere(Vector3f(0.0f, 1.2f, 0.0f), 0.2f, &light));
    scene.camera = Camera::create(Vector3f(0.0f, 1.6f, 1.8f), Vector3f(0, 0, 0),
                                  Vector3f(0, 1, 0), 50.0f, 60.0f);
    scene.camera.init(W, H);
    scene.buildBVH();

    // the medium is carried like the reference's Scene::medium (rendering ignores it)
    scene.medium = Medium::fog();
    scene.medium.bounded = true;
    scene.medium.bounds = Bounds3(Vector3f(-1.0f, -1.0f, -1.0f), Vector3f(1.0f, 1.0f, 1.0f));
    float te = 0.f, tx = 0.f;
    const float c = 0.57735026f; // 1/sqrt(3)
    const bool diag = scene.medium.intersect(Ray(Vector3f(-3.0f), Vector3f(c, c, c)), te, tx);
    std::printf("medium %d %g %g active %d\n", (int) diag, te, tx, (int) scene.medium.active());
    // a direction with zero components: Medium::intersect swaps the slab ends
    // of every axis whose direction is not positive, so this ray misses
    const bool axis = scene.medium.intersect(Ray(Vector3f(0.0f, 0.0f, 3.0f),
                                                 Vector3f(0.0f, 0.0f, -1.0f)), te, tx);
    std::printf("axis-aligned %d\n", (int) axis);

    Integrator integrator(scene, 5, 0.8f);
    RenderSettings settings;
    settings.width = W;
    settings.height = H;
    settings.minSPP = settings.maxSPP = 32;
    settings.seed = 5;
    Renderer r;
    r.Render(scene, integrator, settings);
    std::ofstream(argv[2], std::ios::binary)
        .write((const char *) r.framebuffer().data(), r.framebuffer().size() * sizeof(float));
    return 0;
}
