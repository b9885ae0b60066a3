// Empty stand-in: the reference path that includes it runs its loops serially (TBB disabled).
