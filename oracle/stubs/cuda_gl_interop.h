/* Empty stand-in: the reference includes this OpenGL-interop header but uses
 * nothing from it on the projection path.  Placed first on the include path
 * when oracle/Makefile compiles the reference GPU code headless. */
#pragma once
