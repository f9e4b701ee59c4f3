// Test infrastructure only: the implementations of the vendored stb image
// reader/writer that the reference's EnvMap::load (EnvMap.hpp:35-56) and the
// oracle's .hdr round trip need. In the reference build GLTFLoader.cpp:1-3
// defines them; the oracle leaves the glTF loader out, so this unit does.
#define STB_IMAGE_IMPLEMENTATION
#include "stb_image.h"
#define STB_IMAGE_WRITE_IMPLEMENTATION
#include "stb_image_write.h"
