import sys; p=sys.argv[1].replace('vis.cu','clean.cu'); s=open(p).read()
old='        const bool stage = 2 * sizeof(float) * (size_t)P + 2048 <= (size_t)optin;  // 2 KB: the static arrays'
assert old in s; s=s.replace(old,'        const bool stage = false;'); open(p,'w').write(s)
