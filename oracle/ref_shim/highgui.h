// Empty stand-in for OpenCV 1.x's highgui.h: the reference file that includes it uses nothing from it.
