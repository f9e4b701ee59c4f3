// Uses libprr through the reference-named C++ classes of prr_dropin.hpp: the
// Cornell box of photorealisticrender4610_b200.scenes.cornell_box built with
// MeshTriangle / Sphere / materials / Camera::create, rendered by
// Renderer::Render. Writes the linear framebuffer (floats) to argv[1] and
// prints one Scene::intersect result.
#include "prr_dropin.hpp"

#include <algorithm>

#include <cstdio>
#include <fstream>

static MeshTriangle *quad(Vector3f p0, Vector3f p1, Vector3f p2, Vector3f p3, Material *m) {
    std::vector<Triangle> t = {Triangle(p0, p1, p2, m), Triangle(p0, p2, p3, m)};
    Vector3f lo(std::min({p0.x, p1.x, p2.x, p3.x}), std::min({p0.y, p1.y, p2.y, p3.y}),
                std::min({p0.z, p1.z, p2.z, p3.z}));
    Vector3f hi(std::max({p0.x, p1.x, p2.x, p3.x}), std::max({p0.y, p1.y, p2.y, p3.y}),
                std::max({p0.z, p1.z, p2.z, p3.z}));
    return new MeshTriangle(t, Bounds3(lo, hi), m);
}

int main(int argc, char **argv) {
    const int W = 64, H = 64;
    DiffuseMaterial white, red, green;
    EmissiveMaterial light;
    white.baseColor = Vector3f(0.73f);
    red.baseColor = Vector3f(0.65f, 0.05f, 0.05f);
    green.baseColor = Vector3f(0.12f, 0.45f, 0.15f);
    for (Material *m : {(Material *) &white, (Material *) &red, (Material *) &green}) {
        m->roughness = 1.0f;
        m->metallic = 0.0f;
    }
    light.m_emission = Vector3f(15.0f);
    Scene scene;
    scene.Add(quad({-1, -1, 1}, {1, -1, 1}, {1, -1, -1}, {-1, -1, -1}, &white));
    scene.Add(quad({-1, 1, -1}, {1, 1, -1}, {1, 1, 1}, {-1, 1, 1}, &white));
    scene.Add(quad({-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, &white));
    scene.Add(quad({-1, -1, 1}, {-1, -1, -1}, {-1, 1, -1}, {-1, 1, 1}, &red));
    scene.Add(quad({1, -1, -1}, {1, -1, 1}, {1, 1, 1}, {1, 1, -1}, &green));
    const float y = 0.99f;
    scene.Add(quad({-0.25f, y, -0.25f}, {0.25f, y, -0.25f}, {0.25f, y, 0.25f}, {-0.25f, y, 0.25f},
                   &light));
    scene.Add(new Sphere(Vector3f(-0.4f, -0.7f, -0.3f), 0.3f, &white));
    scene.Add(new Sphere(Vector3f(0.45f, -0.7f, 0.3f), 0.3f, &white));
    scene.camera = Camera::create(Vector3f(0, 0, 3.5f), Vector3f(0, 0, 0), Vector3f(0, 1, 0),
                                  40.0f, 40.0f);
    scene.camera.init(W, H);
    scene.buildBVH();

    Integrator integrator(scene, 5, 0.8f);
    RenderSettings settings;
    settings.width = W;
    settings.height = H;
    settings.minSPP = settings.maxSPP = 16;
    settings.mode = PRR_RENDER_PLAIN;
    settings.exposure = 1.0f;
    Renderer r;
    r.Render(scene, integrator, settings);
    std::ofstream(argv[1], std::ios::binary)
        .write((const char *) r.framebuffer().data(), r.framebuffer().size() * sizeof(float));

    Intersection in = scene.intersect(Ray(Vector3f(0, 0, 3.5f), Vector3f(0, 0, -1)));
    std::printf("hit %d obj %d prim %d t %.6f\n", (int) in.happened, in.object, in.primitive,
                in.tnear);
    Vector3f L = integrator.castRay(Ray(Vector3f(0, 0, 3.5f), Vector3f(0, -0.1f, -1)));
    std::printf("castRay %.6f %.6f %.6f\n", L.x, L.y, L.z);
    return 0;
}
