// Host check of the float32 correctly-rounded exp/log/sin scheme used by the
// GPU kernels: the fast path (a double-precision libm function plus the same
// interval rounding test) and the double-double slow path (ionp_dd.cuh), both
// compared with (float)(long double libm) on every stride-th float32.
// Usage: verify_f32 <0=exp|1=log|2=sin> <slow-path-only 0|1> [stride]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <cstdint>
#include <atomic>
#include <thread>
#include <vector>
#include "ionp_dd.cuh"
using namespace ionp::dd;
static float bf(uint32_t u){float f;memcpy(&f,&u,4);return f;}
static uint32_t fb(float f){uint32_t u;memcpy(&u,&f,4);return u;}
static bool pins(double y, float* out){ const double E=0x1p-49; float a=(float)(y*(1.0-E)), b=(float)(y*(1.0+E)); *out=a; return fb(a)==fb(b);}
static float my_exp(float x, int* slow){ if(x>89.0f) return INFINITY; if(x<-104.0f) return 0.0f; float f; if(pins(exp((double)x),&f)) return f; (*slow)++; return dd_to_float(exp_dd(x)); }
static float my_log(float x, int* slow){ if(x==0) return -INFINITY; if(std::isinf(x)) return x; float f; if(pins(log((double)x),&f)) return f; (*slow)++; return dd_to_float(log_dd(x)); }
static float my_sin(float x, int* slow){ float f; if(pins(sin((double)x),&f)) return f; (*slow)++; return dd_to_float(sin_dd(x)); }
static float slow_only(int w, float x){ if(w==0) return dd_to_float(exp_dd(x)); if(w==1) return dd_to_float(log_dd(x)); return dd_to_float(sin_dd(x)); }
int main(int argc, char** argv){
  int which = atoi(argv[1]); int slowmode = argc > 2 ? atoi(argv[2]) : 0; uint64_t stride = argc > 3 ? strtoull(argv[3], 0, 10) : 1;
  int nt = std::thread::hardware_concurrency();
  std::atomic<uint64_t> n{0}, diff{0}, slow{0};
  std::vector<std::thread> th;
  for(int t=0;t<nt;t++) th.emplace_back([&,t](){
    uint64_t ln=0, ld=0; int ls=0; int printed=0;
    for(uint64_t u=t; u<=0xFFFFFFFFull; u+=nt){
      if ((u % stride) != 0) continue;
      float x=bf((uint32_t)u); if(std::isnan(x) || std::isinf(x)) continue;
      long double r; float mine;
      if(which==0){ if(x>89.0f||x<-104.0f) continue; r=expl((long double)x); mine = slowmode ? slow_only(0,x) : my_exp(x,&ls);} 
      else if(which==1){ if(x<=0) continue; r=logl((long double)x); mine = slowmode ? slow_only(1,x) : my_log(x,&ls);} 
      else { r=sinl((long double)x); mine = slowmode ? slow_only(2,x) : my_sin(x,&ls);} 
      float c=(float)r; ln++;
      if(fb(c)!=fb(mine)){ ld++; if(printed<3){ printed++; printf("DIFF x=%a mine=%a ref=%a\n", x, mine, c);} }
    }
    n+=ln; diff+=ld; slow+=ls;
  });
  for(auto&x:th) x.join();
  printf("which=%d slowmode=%d n=%llu diff=%llu slowpath=%llu\n", which, slowmode, (unsigned long long)n.load(), (unsigned long long)diff.load(), (unsigned long long)slow.load());
}
