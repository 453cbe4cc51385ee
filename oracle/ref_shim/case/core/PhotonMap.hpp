// The reference includes "../core/PhotonMap.hpp" while the file on disk is
// photonmap.hpp (case-insensitive Windows file system); this forwards to it.
#include <core/photonmap.hpp>
