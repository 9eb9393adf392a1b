// Stand-in for the caller's lib/io myio.cpp:12-21 in the drop-in test: records
// argv where libvti_wave.so reads its side channels (data=, gpu=, ...).
int gargc = 0;
char** gargv = nullptr;

void myio_init(int argc, char** argv) {
  gargc = argc;
  gargv = argv;
}
