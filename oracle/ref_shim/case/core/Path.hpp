// Case forward for "../geom/Path.hpp" -> path.hpp (see PhotonMap.hpp).
#include <geom/path.hpp>
