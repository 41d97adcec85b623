// main.cpp -- `rbmd [cuda] -j input.json`: the reference's process entry (main.cpp /
// Application::Run) on the sm_100a library.
#include "app.hpp"

int main(int argc, char** argv) {
  rbmd_host::MDApplication app(argc, argv);
  return app.Run();
}
