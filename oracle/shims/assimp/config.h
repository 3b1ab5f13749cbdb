// Stand-in for the CMake-generated assimp/config.h. The oracle never imports
// models through assimp; the reference's scene module only needs the headers
// to compile. Test infrastructure only.
#pragma once
